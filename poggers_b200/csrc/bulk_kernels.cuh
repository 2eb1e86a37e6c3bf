// bulk_kernels.cuh -- the bulk insert / query / remove kernels behind the C ABI.
//
// One group of G lanes serves one key at a time (the reference launches one
// tile per key, tables/base_table.cuh:321-329); a grid sized to the resident
// capacity walks the batch in a grid-stride loop, so the launch costs are
// the same for 1k and 1G keys.  Keys and values are read once, coalesced;
// results are written once, coalesced; counters are warp-aggregated.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "poggers_b200/level.cuh"

namespace pg {

enum bulk_op : int { OP_INSERT = 0, OP_QUERY = 1, OP_REMOVE = 2 };

struct bulk_args {
    const uint64_t *keys;
    const void *vals_in;
    void *vals_out;
    uint8_t *flags;                 // ok / found
    unsigned long long *count;      // fail count (insert) or hit count (query / remove)
    uint64_t n;
    // insert over a permuted copy of the batch: flags were preset to 1 and only
    // a failure is written, at flags[perm[i]] (the key's place in the caller's batch)
    const uint32_t *perm;
    // the permuted copy in runs of region_cap entries, one run per table region:
    // run r holds region_cursor[r] - r * region_cap keys (at most region_cap),
    // the rest of the run is unused; region_div = 2^64 / region_cap rounded up,
    // so that i / region_cap = mulhi(region_div, i) for i < 2^32
    const unsigned long long *region_cursor;
    uint64_t region_cap, region_div;
    // insert only the keys whose bit is set (those that did not fit their run)
    const uint32_t *only;
};

__device__ __forceinline__ void add_count(unsigned long long *count, uint32_t c)
{
    if (!count) return;
    unsigned am = __activemask();
    unsigned s = __reduce_add_sync(am, c);
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(am) - 1) && s) atomicAdd(count, (unsigned long long)s);
}

// Minimum resident 256-thread blocks per SM the register allocation must allow
// (8 = full occupancy at 32 registers); a build-time knob measured by the tuner.
#ifndef PG_MIN_BLOCKS
#define PG_MIN_BLOCKS 1
#endif

// The fingerprint walk is latency-bound on L2 round trips: full occupancy (8
// blocks of 256, 32 registers) measured 7 % faster on the region-ordered
// insert at 2^26 slots despite a few bytes of spill (and 6 blocks, 40
// registers, 6 % slower on the insert kernel again after later changes).
#ifndef PG_FP_MIN_BLOCKS
#define PG_FP_MIN_BLOCKS 8
#endif
// The filters' kernels (16-bit tags) are bound by random sector reads and
// need many keys in flight: held to 6 resident blocks of 256 (40 registers,
// a few spilled words) they ran 1.2-1.4x faster than at their natural 93-103
// registers (2 blocks).
#ifndef PG_FILTER_MIN_BLOCKS
#define PG_FILTER_MIN_BLOCKS 6
#endif
// Only the one-lane filter kernels (large tables) are held: the 4-lane ones
// serve two-choice levels below 2^18 slots, which launch few blocks anyway,
// and at 40 registers they would spill ~0.7 KB per thread.
template <int FMT, int G = 1>
constexpr int min_blocks_of()
{
    if (FMT == FMT_KV64_FP) return PG_FP_MIN_BLOCKS;
    if ((FMT == FMT_TAGVAL16 || FMT == FMT_TAGVAL16_SPLIT || FMT == FMT_TAG16) && G == 1) return PG_FILTER_MIN_BLOCKS;
    return PG_MIN_BLOCKS;
}

template <int FMT, int B, int G, int S0, bool BK, int OP>
__global__ void __launch_bounds__(256, min_blocks_of<FMT, G>()) k_bulk(table_desc t, bulk_args a)
{
    using F = fmt_t<FMT>;
    using V = typename F::V;
    using T = table_ops<FMT, B, G, S0, BK>;
    const group<G> g = group<G>::make();
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
    const V *vin = static_cast<const V *>(a.vals_in);
    V *vout = static_cast<V *>(a.vals_out);
    uint32_t c = 0;
    if constexpr (OP == OP_INSERT) {
        if (a.only) {
            // the keys a region-sorted pass could not place in their runs, in batch order
            const uint64_t nw = (a.n + 31) / 32;
            for (uint64_t w = gid; w < nw; w += ngroups) {
                uint32_t bits = __ldg(a.only + w);
                while (bits) {
                    const uint64_t i = w * 32 + (uint64_t)(__ffs(bits) - 1);
                    bits &= bits - 1;
                    const bool r = T::insert(t, g, __ldg(a.keys + i), vin ? __ldg(vin + i) : (V)0);
                    if (g.gl == 0) {
                        if (a.flags) a.flags[i] = (uint8_t)r;
                        c += !r;
                    }
                }
            }
            add_count(a.count, c);
            return;
        }
    }
    for (uint64_t i = gid; i < a.n; i += ngroups) {
        if constexpr (OP == OP_INSERT) {
            if (a.region_cap) {
                // past the keys of this region's run: nothing there
                const uint64_t r = __umul64hi(a.region_div, i);
                if (i - r * a.region_cap >= a.region_cursor[r] - r * a.region_cap) continue;
            }
        }
        const uint64_t key = __ldg(a.keys + i);
        bool r;
        if constexpr (OP == OP_INSERT) {
            V v = vin ? __ldg(vin + i) : (V)0;
            r = T::insert(t, g, key, v);
            if (g.gl == 0) {
                if (a.flags) {
                    if (!a.perm) __stcs(a.flags + i, (uint8_t)r);
                    else if (!r) a.flags[a.perm[i]] = 0;
                }
                c += !r;
            }
        } else if constexpr (OP == OP_QUERY) {
            V v = 0;
            r = T::query(t, g, key, v);
            if (g.gl == 0) {
                if (vout) __stcs(vout + i, r ? v : (V)0);
                if (a.flags) __stcs(a.flags + i, (uint8_t)r);
                c += r;
            }
        } else {
            r = T::remove(t, g, key);
            if (g.gl == 0) {
                if (a.flags) __stcs(a.flags + i, (uint8_t)r);
                c += r;
            }
        }
    }
    add_count(a.count, c);
}

template <int FMT, int B, int G, int S0, bool BK>
cudaError_t launch_bgs(int op, const table_desc &t, const bulk_args &a, dim3 grid, dim3 block, cudaStream_t s)
{
    switch (op) {
    case OP_INSERT: k_bulk<FMT, B, G, S0, BK, OP_INSERT><<<grid, block, 0, s>>>(t, a); break;
    case OP_QUERY: k_bulk<FMT, B, G, S0, BK, OP_QUERY><<<grid, block, 0, s>>>(t, a); break;
    default: k_bulk<FMT, B, G, S0, BK, OP_REMOVE><<<grid, block, 0, s>>>(t, a); break;
    }
    return cudaGetLastError();
}

// the primary level's scheme and the presence of a backing level are
// compile-time, so a single-level table carries no backing-path code
template <int FMT, int B, int G>
cudaError_t launch_bg(int op, const table_desc &t, const bulk_args &a, dim3 grid, dim3 block, cudaStream_t s)
{
    const bool bk = t.nlevels > 1;
    if (t.lv[0].scheme == SCHEME_BUCKET)
        return bk ? launch_bgs<FMT, B, G, SCHEME_BUCKET, true>(op, t, a, grid, block, s)
                  : launch_bgs<FMT, B, G, SCHEME_BUCKET, false>(op, t, a, grid, block, s);
    return bk ? launch_bgs<FMT, B, G, SCHEME_TWO_CHOICE, true>(op, t, a, grid, block, s)
              : launch_bgs<FMT, B, G, SCHEME_TWO_CHOICE, false>(op, t, a, grid, block, s);
}

template <int FMT, int B>
cudaError_t launch_b(int op, uint32_t tile, const table_desc &t, const bulk_args &a, dim3 grid, dim3 block,
                     cudaStream_t s)
{
    switch (tile) {
    case 1: return launch_bg<FMT, B, 1>(op, t, a, grid, block, s);
    case 2: return launch_bg<FMT, B, 2>(op, t, a, grid, block, s);
    case 4: return launch_bg<FMT, B, 4>(op, t, a, grid, block, s);
    case 8:
        if constexpr (B >= 8) return launch_bg<FMT, B, 8>(op, t, a, grid, block, s);
        else return cudaErrorInvalidConfiguration;
    case 16:
        if constexpr (B >= 16) return launch_bg<FMT, B, 16>(op, t, a, grid, block, s);
        else return cudaErrorInvalidConfiguration;
    default: return cudaErrorInvalidConfiguration;
    }
}

template <int FMT>
cudaError_t launch_fmt(int op, uint32_t bucket, uint32_t tile, const table_desc &t, const bulk_args &a,
                       dim3 grid, dim3 block, cudaStream_t s)
{
    switch (bucket) {
    case 4: return launch_b<FMT, 4>(op, tile, t, a, grid, block, s);
    case 8: return launch_b<FMT, 8>(op, tile, t, a, grid, block, s);
    case 16: return launch_b<FMT, 16>(op, tile, t, a, grid, block, s);
    case 32: return launch_b<FMT, 32>(op, tile, t, a, grid, block, s);
    default: return cudaErrorInvalidConfiguration;
    }
}

// one per internal format, compiled in separate translation units
#define PG_DECLARE_LAUNCH(name)                                                                                   \
    cudaError_t name(int op, uint32_t bucket, uint32_t tile, const table_desc &t, const bulk_args &a, dim3 grid, \
                     dim3 block, cudaStream_t s)
PG_DECLARE_LAUNCH(launch_kv64);
PG_DECLARE_LAUNCH(launch_kv64_split);
PG_DECLARE_LAUNCH(launch_tagval16);
PG_DECLARE_LAUNCH(launch_tagval16_split);
PG_DECLARE_LAUNCH(launch_tag16);
PG_DECLARE_LAUNCH(launch_kv64_fp);

}  // namespace pg
