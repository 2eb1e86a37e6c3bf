// partition.cu -- region-ordered bulk insert for large batches into large
// uint64 tables.
//
// A random insert into a table much larger than L2 costs a DRAM read for its
// CAS (with fingerprints, a sector the slot store only partly writes) and a
// DRAM write-back of the dirty sector, per key: random DRAM transactions are
// the limit.  Sorting the batch by the table region of each
// key's first bucket (a counting sort into R regions that each fit in L2) lets
// the insert kernel sweep the table region by region: while the resident
// threads work through one region, its lines stay in L2, so a line is
// fetched once and written back once for all the keys that land in it (about
// seven at 0.9 load with 8-slot buckets) instead of once per key.  Keys whose
// first bucket is full still probe at random.
//
// The per-key work is the ordinary insert; only the order in which a launch
// visits the keys changes, and concurrent inserts have no defined order in
// the reference either.  The caller's ok flags are preset to 1 and a failed
// insert clears its flag through the permutation.
#include <math.h>
#include <stdint.h>
#include <cuda_runtime.h>

#include "poggers_b200.h"
#include "bulk_kernels.cuh"
#include "table_internal.h"

namespace pg {

constexpr uint32_t kPartThreads = 256;
constexpr uint32_t kPartPerThread = 4;
constexpr uint32_t kPartTile = kPartThreads * kPartPerThread;  // keys per scatter tile
constexpr uint32_t kPartMaxRegions = 1024;
static_assert(kPartTile <= 65536 && kPartMaxRegions <= 65536, "a staged entry's tag packs region and index in 16 bits each");
#ifndef PG_PART_REGION_MB
#define PG_PART_REGION_MB 32
#endif
constexpr uint64_t kPartRegionBytes = (uint64_t)PG_PART_REGION_MB << 20;  // table bytes per region (a power of two)
constexpr uint64_t kPartMinKeys = 1ull << 20;         // smaller batches insert unsorted
#ifndef PG_PART_WIDE
#define PG_PART_WIDE 1  // build knob: 0 keeps the 1024-key tiles at any region count
#endif

// region of a key = its first bucket >> shift: regions are runs of 2^shift buckets
struct region_router {
    level_desc L;
    uint32_t shift;
    __device__ __forceinline__ uint32_t operator()(uint64_t key) const
    {
        return (uint32_t)(L.nbmod.mod(murmur64a_u64(key, L.seed)) >> shift);
    }
};

// owner of a key among nshards shards: the high bits of a routing hash
// (multiply-shift, so owners are uniform for any shard count)
struct shard_router {
    uint64_t seed;
    uint32_t nshards;
    __device__ __forceinline__ uint32_t operator()(uint64_t key) const
    {
        return (uint32_t)umulhi64(murmur64a_u64(key, seed), nshards);
    }
};

template <class Router>
__global__ void __launch_bounds__(kPartThreads) k_part_count(Router route, const uint64_t *keys, uint64_t n,
                                                             uint32_t R, unsigned long long *counts)
{
    __shared__ unsigned int hist[kPartMaxRegions];
    for (uint32_t r = threadIdx.x; r < R; r += blockDim.x) hist[r] = 0;
    __syncthreads();
    // kPartPerThread keys per thread per round, all loads issued before any is used
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * kPartPerThread) {
        uint64_t k[kPartPerThread];
#pragma unroll
        for (uint32_t j = 0; j < kPartPerThread; j++) {
            const uint64_t i = i0 + j * stride;
            k[j] = i < n ? __ldcs(keys + i) : 0;
        }
#pragma unroll
        for (uint32_t j = 0; j < kPartPerThread; j++)
            if (i0 + j * stride < n) atomicAdd(&hist[route(k[j])], 1u);
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < R; r += blockDim.x)
        if (hist[r]) atomicAdd(counts + r, (unsigned long long)hist[r]);
}

// exclusive prefix sum of the R region counts into the cursors (one warp)
__global__ void k_part_scan(const unsigned long long *counts, unsigned long long *cursors, uint32_t R)
{
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long carry = 0;
    for (uint32_t r0 = 0; r0 < R; r0 += 32) {
        const uint32_t r = r0 + lane;
        const unsigned long long c = r < R ? counts[r] : 0ULL;
        unsigned long long x = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= (uint32_t)d) x += y;
        }
        if (r < R) cursors[r] = carry + x - c;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
}

// cursors[r] = r * cap: the start of region r's run of cap entries
__global__ void k_part_bases(unsigned long long *cursors, uint32_t R, uint64_t cap)
{
    for (uint32_t r = threadIdx.x; r < R; r += blockDim.x) cursors[r] = (unsigned long long)r * cap;
}

// One tile of kPartTile keys at a time: count the tile's keys per region in
// shared memory, reserve one run per region from the global cursors, sort the
// tile by region in shared memory, then write each region's run with
// consecutive threads on consecutive addresses.  With cap != 0 region r owns
// the cap entries from r * cap; a key reserved past them is not written and
// its bit (by its index in the batch) is set in ovf instead.
// The per-region arrays take part_scatter_smem(R) bytes of dynamic shared
// memory beside the 20 KB of staged entries (more resident blocks, forced by
// register limits of 40 or 32, measured 2 % slower).  Tiles of 4 keys per
// thread: 2 measured 9 % slower for the whole insert call, 8 the same (ncu:
// issue-bound with barrier and shared-memory stalls at 45 % of DRAM peak, not
// bound by DRAM).  Staging key and value as one 16-byte entry with region and
// index packed in one word, and each region's output offset computed once per
// tile, took the kernel from 534 to 500 us at 2^26 slots.
inline size_t part_scatter_smem(uint32_t R) { return (size_t)R * (sizeof(unsigned long long) + 2 * sizeof(unsigned)); }

// a key and its value staged in shared memory (one 16-byte access each way)
template <class V>
struct __align__(16) part_entry {
    uint64_t k;
    V v;
};

template <class Router, class V>
__global__ void __launch_bounds__(kPartThreads)
    k_part_scatter(Router route, const uint64_t *keys, const V *vals, uint64_t n, uint32_t R,
                   unsigned long long *cursors, uint64_t *okeys, V *ovals, uint32_t *operm, uint64_t cap,
                   uint32_t *ovf)
{
    extern __shared__ unsigned long long part_dyn[];
    // per region: the reservation, then (once the tile is sorted) the offset
    // from a tile position to its place in the output, gbase - lstart
    unsigned long long *gbase = part_dyn;
    unsigned int *cnt = reinterpret_cast<unsigned int *>(gbase + R);      // R tile counts
    unsigned int *lstart = cnt + R;                                       // R tile offsets
    __shared__ part_entry<V> skv[kPartTile];
    __shared__ uint32_t stag[kPartTile];  // region << 16 | the entry's index in the tile
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    for (uint64_t t0 = (uint64_t)blockIdx.x * kPartTile; t0 < n; t0 += (uint64_t)gridDim.x * kPartTile) {
        const uint32_t tn = (uint32_t)((n - t0) < kPartTile ? (n - t0) : kPartTile);
        for (uint32_t r = tid; r < R; r += blockDim.x) cnt[r] = 0;
        __syncthreads();
        uint64_t k[kPartPerThread];
        V v[kPartPerThread];
        uint32_t reg[kPartPerThread], rank[kPartPerThread];
#pragma unroll
        for (uint32_t j = 0; j < kPartPerThread; j++) {
            const uint32_t e = j * kPartThreads + tid;
            if (e < tn) {
                k[j] = __ldcs(keys + t0 + e);
                v[j] = ovals ? vals[t0 + e] : (V)0;
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < kPartPerThread; j++) {
            const uint32_t e = j * kPartThreads + tid;
            reg[j] = 0xFFFFFFFFu;
            if (e < tn) {
                reg[j] = route(k[j]);
                rank[j] = atomicAdd(&cnt[reg[j]], 1u);
            }
        }
        __syncthreads();
        // tile-local exclusive scan of cnt (warp 0) and the global reservations (all threads)
        if (warp == 0) {
            unsigned int carry = 0;
            for (uint32_t r0 = 0; r0 < R; r0 += 32) {
                const uint32_t r = r0 + lane;
                const unsigned int c = r < R ? cnt[r] : 0u;
                unsigned int x = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const unsigned int y = __shfl_up_sync(0xffffffffu, x, d);
                    if (lane >= (uint32_t)d) x += y;
                }
                if (r < R) lstart[r] = carry + x - c;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
        }
        for (uint32_t r = tid; r < R; r += blockDim.x)
            if (cnt[r]) gbase[r] = atomicAdd(cursors + r, (unsigned long long)cnt[r]);
        __syncthreads();
#pragma unroll
        for (uint32_t j = 0; j < kPartPerThread; j++) {
            if (reg[j] == 0xFFFFFFFFu) continue;
            const uint32_t e = j * kPartThreads + tid;
            const uint32_t at = lstart[reg[j]] + rank[j];
            skv[at] = part_entry<V>{k[j], v[j]};
            stag[at] = (reg[j] << 16) | e;
        }
        // the regions' offsets from tile position to output place (wraps mod 2^64 when lstart > gbase)
        for (uint32_t r = tid; r < R; r += blockDim.x)
            if (cnt[r]) gbase[r] -= lstart[r];
        __syncthreads();
        for (uint32_t e = tid; e < tn; e += blockDim.x) {
            const uint32_t tag = stag[e];
            const uint32_t r = tag >> 16;
            const uint32_t src = (uint32_t)t0 + (tag & 0xFFFFu);
            const uint64_t pos = gbase[r] + e;
            if (cap && pos >= (uint64_t)(r + 1) * cap) {
                atomicOr(ovf + (src >> 5), 1u << (src & 31u));
                continue;
            }
            const part_entry<V> kv = skv[e];
            okeys[pos] = kv.k;
            if (ovals) ovals[pos] = kv.v;
            operm[pos] = src;
        }
        __syncthreads();
    }
}

// Many regions (large tables): a 1024-key tile then holds only a few keys per
// region, so each run it writes is a sector or less and the writes coalesce
// poorly.  This variant takes tiles of kWideTile keys (512 threads, 8 keys
// each), kept in dynamic shared memory in the order they arrive with their
// region and rank; only a 2-byte index is sorted by region, and the runs are
// then written by consecutive threads from it.  Its dynamic shared memory is
// part_scatter_wide_smem(R) bytes (106 KB at 1024 regions: two blocks per SM).
// Measured: the insert call at 2^29 slots (256 regions) 27.98 -> 23.19 ms, at
// 2^30 slots (512 regions, 966 M keys) 66.7 -> 51.1 ms.
constexpr uint32_t kWideThreads = 512;
constexpr uint32_t kWidePerThread = 8;
constexpr uint32_t kWideTile = kWideThreads * kWidePerThread;
constexpr uint32_t kWideMinRegions = 65;  // tables of more than 64 regions take this variant
static_assert(kWideTile <= 65536, "ranks and indices of a wide tile fit 16 bits");
inline size_t part_scatter_wide_smem(uint32_t R)
{
    return (size_t)R * 16 + (size_t)kWideTile * (sizeof(part_entry<unsigned long long>) + 4 + 2);
}

template <class Router, class V>
__global__ void __launch_bounds__(kWideThreads)
    k_part_scatter_wide(Router route, const uint64_t *keys, const V *vals, uint64_t n, uint32_t R,
                        unsigned long long *cursors, uint64_t *okeys, V *ovals, uint32_t *operm, uint64_t cap,
                        uint32_t *ovf)
{
    extern __shared__ unsigned long long part_dyn[];
    unsigned long long *gbase = part_dyn;                                       // R: reservation, then offset
    unsigned int *cnt = reinterpret_cast<unsigned int *>(gbase + R);            // R tile counts
    unsigned int *lstart = cnt + R;                                             // R tile offsets
    part_entry<V> *akv = reinterpret_cast<part_entry<V> *>(lstart + R);         // kWideTile, arrival order
    uint32_t *atag = reinterpret_cast<uint32_t *>(akv + kWideTile);             // region << 16 | rank
    uint16_t *sidx = reinterpret_cast<uint16_t *>(atag + kWideTile);            // sorted: arrival index
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    for (uint64_t t0 = (uint64_t)blockIdx.x * kWideTile; t0 < n; t0 += (uint64_t)gridDim.x * kWideTile) {
        const uint32_t tn = (uint32_t)((n - t0) < kWideTile ? (n - t0) : kWideTile);
        for (uint32_t r = tid; r < R; r += blockDim.x) cnt[r] = 0;
        __syncthreads();
        uint64_t k[kWidePerThread];
        V v[kWidePerThread];
#pragma unroll
        for (uint32_t j = 0; j < kWidePerThread; j++) {
            const uint32_t e = j * kWideThreads + tid;
            if (e < tn) {
                k[j] = __ldcs(keys + t0 + e);
                v[j] = ovals ? vals[t0 + e] : (V)0;
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < kWidePerThread; j++) {
            const uint32_t e = j * kWideThreads + tid;
            if (e < tn) {
                const uint32_t reg = route(k[j]);
                const uint32_t rank = atomicAdd(&cnt[reg], 1u);
                akv[e] = part_entry<V>{k[j], v[j]};
                atag[e] = (reg << 16) | rank;
            }
        }
        __syncthreads();
        if (warp == 0) {
            unsigned int carry = 0;
            for (uint32_t r0 = 0; r0 < R; r0 += 32) {
                const uint32_t r = r0 + lane;
                const unsigned int c = r < R ? cnt[r] : 0u;
                unsigned int x = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const unsigned int y = __shfl_up_sync(0xffffffffu, x, d);
                    if (lane >= (uint32_t)d) x += y;
                }
                if (r < R) lstart[r] = carry + x - c;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
        }
        for (uint32_t r = tid; r < R; r += blockDim.x)
            if (cnt[r]) gbase[r] = atomicAdd(cursors + r, (unsigned long long)cnt[r]);
        __syncthreads();
        for (uint32_t e = tid; e < tn; e += blockDim.x) {
            const uint32_t tag = atag[e];
            sidx[lstart[tag >> 16] + (tag & 0xFFFFu)] = (uint16_t)e;
        }
        for (uint32_t r = tid; r < R; r += blockDim.x)
            if (cnt[r]) gbase[r] -= lstart[r];
        __syncthreads();
        for (uint32_t q = tid; q < tn; q += blockDim.x) {
            const uint32_t e = sidx[q];
            const uint32_t r = atag[e] >> 16;
            const uint32_t src = (uint32_t)t0 + e;
            const uint64_t pos = gbase[r] + q;
            if (cap && pos >= (uint64_t)(r + 1) * cap) {
                atomicOr(ovf + (src >> 5), 1u << (src & 31u));
                continue;
            }
            const part_entry<V> kv = akv[e];
            okeys[pos] = kv.k;
            if (ovals) ovals[pos] = kv.v;
            operm[pos] = src;
        }
        __syncthreads();
    }
}

}  // namespace pg

using namespace pg;

// Called by pg_bulk_insert with the caller's batch in `a`.  When the batch
// qualifies it writes the region-ordered copy into the table's scratch,
// presets the ok flags to 1, points `a` at the copy (in runs, one per region)
// and returns true; the caller then runs the ordinary insert launch on `a`,
// and after it the keys that did not fit their run, from the caller's batch
// (bits in a.only, returned through `only`).  Returns false (and leaves `a`
// alone) when the batch should take the ordinary path: partitioning off, a
// serial launch shape, not a uint64 bucket table, table or batch too small
// for the sort to pay, or no memory for the scratch.
//
// The runs have a fixed capacity: the keys expected in a full region (the
// first bucket is MurmurHash64A % nb, uniform over the buckets) plus eight
// standard deviations and 1024, so the sort needs no counting pass.  Only a
// batch far from uniform over the table (many copies of one key, say) fills
// a run; its extra keys are inserted by the second pass, in batch order.
namespace {

// The sort's plan for a batch of n keys: regions of 2^shift buckets (about
// kPartRegionBytes of slots each, at most kPartMaxRegions), run capacity, the
// entries of the sorted copy and the scratch bytes.  False when the batch
// takes the ordinary path.
struct region_plan {
    uint32_t shift, R;
    uint64_t cap, nv, cur_off, ovf_off, need;
};

bool plan_regions(const pg_table *t, uint64_t n, region_plan &pl)
{
    if (t->bytes[0] < 2 * kPartRegionBytes || n < kPartMinKeys || n >= (1ull << 32)) return false;
    const uint64_t nb = t->desc.lv[0].nbmod.d, bucket_bytes = t->bytes[0] / nb;
    uint32_t shift = 0;
    while ((bucket_bytes << (shift + 1)) <= kPartRegionBytes) shift++;
    while (((nb - 1) >> shift) + 1 > kPartMaxRegions) shift++;
    const uint32_t R = (uint32_t)(((nb - 1) >> shift) + 1);
    const double expect = (double)n * (double)(1ull << shift) / (double)nb;
    pl.shift = shift;
    pl.R = R;
    pl.cap = (uint64_t)(expect + 8.0 * sqrt(expect)) + 1024;
    pl.nv = pl.cap * R;  // entries of the sorted copy, runs included
    if (pl.nv >= (1ull << 32)) return false;
    // scratch: keys (8 B), values (8 B) and original index (4 B) per entry;
    // run cursors; one overflow bit per key of the batch
    pl.cur_off = (pl.nv * 20 + 255) & ~255ull;
    pl.ovf_off = pl.cur_off + ((R * 8ull + 255) & ~255ull);
    pl.need = pl.ovf_off + ((n + 31) / 32) * 4;
    return true;
}

// Grow the table's sort scratch to `need` bytes, ordered on stream s (a
// stream-ordered free and allocation: no device-wide synchronization).
bool grow_scratch(pg_table *t, uint64_t need, cudaStream_t s)
{
    if (t->part_bytes >= need) return true;
    if (t->part_buf) cudaFreeAsync(t->part_buf, s);
    t->part_buf = nullptr;
    t->part_bytes = 0;
    if (cudaMallocAsync(&t->part_buf, need, s) != cudaSuccess) {
        cudaGetLastError();
        t->part_buf = nullptr;
        return false;
    }
    t->part_bytes = need;
    return true;
}

bool region_sort(pg_table *t, bulk_args &a, const uint32_t *&only, cudaStream_t s)
{
    const uint64_t n = a.n;
    region_plan pl;
    if (!plan_regions(t, n, pl)) return false;
    if (!grow_scratch(t, pl.need, s)) return false;
    const uint32_t shift = pl.shift, R = pl.R;
    const uint64_t cap = pl.cap, nv = pl.nv, cur_off = pl.cur_off, ovf_off = pl.ovf_off;
    unsigned char *p = static_cast<unsigned char *>(t->part_buf);
    uint64_t *okeys = reinterpret_cast<uint64_t *>(p);
    void *ovals = a.vals_in ? static_cast<void *>(p + nv * 8) : nullptr;
    uint32_t *operm = reinterpret_cast<uint32_t *>(p + nv * 16);
    unsigned long long *cursors = reinterpret_cast<unsigned long long *>(p + cur_off);
    uint32_t *ovf = reinterpret_cast<uint32_t *>(p + ovf_off);
    const unsigned grid = (unsigned)(t->num_sms * 8);
    cudaMemsetAsync(ovf, 0, ((n + 31) / 32) * 4, s);
    k_part_bases<<<1, kPartThreads, 0, s>>>(cursors, R, cap);
    const region_router route{t->desc.lv[0], shift};
    if (R >= kWideMinRegions && PG_PART_WIDE) {
        const size_t smem = part_scatter_wide_smem(R);
        auto *fn = k_part_scatter_wide<region_router, unsigned long long>;
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return false;  // not expected on sm_100a; the batch then takes the ordinary path
        }
        fn<<<(unsigned)(t->num_sms * 2), kWideThreads, smem, s>>>(
            route, a.keys, static_cast<const unsigned long long *>(a.vals_in), n, R, cursors, okeys,
            static_cast<unsigned long long *>(ovals), operm, cap, ovf);
    } else {
        k_part_scatter<<<grid, kPartThreads, part_scatter_smem(R), s>>>(
            route, a.keys, static_cast<const unsigned long long *>(a.vals_in), n, R, cursors, okeys,
            static_cast<unsigned long long *>(ovals), operm, cap, ovf);
    }
    if (a.flags) cudaMemsetAsync(a.flags, 1, n, s);
    a.keys = okeys;
    a.vals_in = ovals;
    a.perm = operm;
    a.n = nv;
    a.region_cursor = cursors;
    a.region_cap = cap;
    a.region_div = ~0ull / cap + 1;
    only = ovf;
    return true;
}

}  // namespace

bool pg_partition_reserve(pg_table *t, uint64_t max_keys, cudaStream_t s)
{
    region_plan pl;
    if (!plan_regions(t, max_keys, pl)) return true;  // such batches take the ordinary path: nothing to reserve
    return grow_scratch(t, pl.need, s);
}

bool pg_partition_insert(pg_table *t, bulk_args &a, const uint32_t *&only, cudaStream_t s)
{
    const bool kv64 = t->ifmt == FMT_KV64 || t->ifmt == FMT_KV64_SPLIT || t->ifmt == FMT_KV64_FP;
    if (!t->partition || !kv64 || t->cfg.levels[0].scheme != PG_SCHEME_BUCKET || t->max_blocks == 1) return false;
    return region_sort(t, a, only, s);
}

// ---------------------------------------------------------------- sharding
// Routing of a batch to the shards of a table partitioned over several GPUs:
// the same counting sort, by owner instead of by region.

namespace pg {

template <class V>
__global__ void __launch_bounds__(256) k_scatter_by_perm(const V *src, const uint32_t *perm, uint64_t n, V *dst)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[perm[i]] = src[i];
}

namespace {

template <class V>
pg_status route_t(const uint64_t *keys, const void *vals, uint64_t n, uint32_t nshards, uint64_t seed,
                  uint64_t *okeys, void *ovals, uint32_t *operm, uint64_t *counts, cudaStream_t s, unsigned grid)
{
    const shard_router route{seed, nshards};
    unsigned long long *c = reinterpret_cast<unsigned long long *>(counts);
    unsigned long long *cur = c + nshards;
    if (cudaMemsetAsync(c, 0, nshards * sizeof(unsigned long long), s) != cudaSuccess) return PG_ERR_CUDA;
    k_part_count<<<grid, kPartThreads, 0, s>>>(route, keys, n, nshards, c);
    k_part_scan<<<1, 32, 0, s>>>(c, cur, nshards);
    k_part_scatter<<<grid, kPartThreads, part_scatter_smem(nshards), s>>>(
        route, keys, static_cast<const V *>(vals), n, nshards, cur, okeys, static_cast<V *>(ovals), operm, 0, nullptr);
    return cudaGetLastError() == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

int sm_count()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 148;
    }
    return sms;
}

}  // namespace

}  // namespace pg

extern "C" {

uint32_t pg_host_shard_of(uint64_t key, uint64_t route_seed, uint32_t nshards)
{
    if (nshards == 0) return 0;
    return (uint32_t)pg::umulhi64(pg::murmur64a_u64(key, route_seed), nshards);
}

pg_status pg_route_by_shard(const uint64_t *d_keys, const void *d_vals, uint32_t val_bytes, uint64_t n,
                            uint32_t nshards, uint64_t route_seed, uint64_t *d_keys_out, void *d_vals_out,
                            uint32_t *d_perm_out, uint64_t *d_counts, pg_stream_t stream)
{
    if (nshards == 0 || nshards > pg::kPartMaxRegions || !d_counts) return PG_ERR_INVALID;
    if (n >= (1ull << 32)) return PG_ERR_INVALID;
    if (!(val_bytes == 0 || val_bytes == 1 || val_bytes == 2 || val_bytes == 8)) return PG_ERR_INVALID;
    if (val_bytes && (!d_vals) != (!d_vals_out)) return PG_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) {
        return cudaMemsetAsync(d_counts, 0, nshards * sizeof(uint64_t), s) == cudaSuccess ? PG_OK : PG_ERR_CUDA;
    }
    if (!d_keys || !d_keys_out || !d_perm_out) return PG_ERR_INVALID;
    const unsigned grid = (unsigned)(pg::sm_count() * 8);
    const void *v = val_bytes ? d_vals : nullptr;
    void *vo = val_bytes ? d_vals_out : nullptr;
    switch (val_bytes) {
    case 8: return pg::route_t<unsigned long long>(d_keys, v, n, nshards, route_seed, d_keys_out, vo, d_perm_out,
                                                   d_counts, s, grid);
    case 2: return pg::route_t<unsigned short>(d_keys, v, n, nshards, route_seed, d_keys_out, vo, d_perm_out,
                                               d_counts, s, grid);
    case 1: return pg::route_t<unsigned char>(d_keys, v, n, nshards, route_seed, d_keys_out, vo, d_perm_out,
                                              d_counts, s, grid);
    default: return pg::route_t<unsigned long long>(d_keys, nullptr, n, nshards, route_seed, d_keys_out, nullptr,
                                                    d_perm_out, d_counts, s, grid);
    }
}

pg_status pg_scatter_by_perm(const void *d_src, const uint32_t *d_perm, uint64_t n, uint32_t elem_bytes, void *d_dst,
                             pg_stream_t stream)
{
    if (n == 0) return PG_OK;
    if (!d_src || !d_perm || !d_dst) return PG_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned grid = (unsigned)(pg::sm_count() * 8);
    switch (elem_bytes) {
    case 1: pg::k_scatter_by_perm<unsigned char><<<grid, 256, 0, s>>>(static_cast<const unsigned char *>(d_src), d_perm, n, static_cast<unsigned char *>(d_dst)); break;
    case 2: pg::k_scatter_by_perm<unsigned short><<<grid, 256, 0, s>>>(static_cast<const unsigned short *>(d_src), d_perm, n, static_cast<unsigned short *>(d_dst)); break;
    case 8: pg::k_scatter_by_perm<unsigned long long><<<grid, 256, 0, s>>>(static_cast<const unsigned long long *>(d_src), d_perm, n, static_cast<unsigned long long *>(d_dst)); break;
    default: return PG_ERR_INVALID;
    }
    return cudaGetLastError() == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

}  // extern "C"
