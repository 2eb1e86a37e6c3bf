// batch_kernels.cuh -- many tables, many requests, one persistent launch.
//
// The reference serves one table per launch (its drivers launch one kernel
// per batch per table, tests/src/test_mhm_tcf.cu:603-685).  For many small
// tables of uneven size that is launch-bound, so here a batch of requests
// {table, op, key offset, key count} over any number of registered tables is
// served by two kernels:
//   k_batch_plan: one block prefix-sums the requests' chunk counts into
//                 chunk_start[] and zeroes the work counter (both scratch);
//   k_batch:      a persistent grid whose warps claim chunks of CHUNK keys with
//                 one atomicAdd each, find the chunk's request by binary
//                 search, and run the same per-key group code as the bulk
//                 kernels against that request's table.
// The request count is read from device memory, so the pair can be captured
// in a CUDA graph once and replayed with other batches.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "poggers_b200.h"
#include "bulk_kernels.cuh"

namespace pg {

constexpr uint32_t kBatchChunk = 256;  // keys per claimed chunk

struct batch_args {
    const table_desc *tables;
    const pg_op_desc *ops;
    const uint32_t *nops;          // device: number of requests
    unsigned long long *chunk_start;  // scratch: max_ops + 1 entries
    unsigned long long *work;         // scratch: chunk counter
    const uint64_t *keys;
    const void *vals_in;
    void *vals_out;
    uint8_t *flags;
    unsigned long long *op_counts;    // per request: hits (query / remove) or failures (insert)
    uint32_t max_ops;
    uint32_t ntables;
};

// Keys per chunk of a request.  Warps claim chunks in request order, so the
// chunks in flight at once can cover every key of a table: a 2^20-slot TCF
// (65,536 buckets) would have some 14 keys per bucket in flight, whose claims
// contend and whose fill checks see the bucket before the others land.  An
// insert request therefore gets at most one chunk per PG_BATCH_INSERT_BUCKETS
// of its primary level's buckets (bigger chunks, each a warp's sequential
// work); queries and removes keep kBatchChunk.  0 turns the cap off.
// Measured on config 3 (1024 TCFs of 2^12-2^20 slots, graph replay of the
// insert and query runs): no cap 13.21 ms, one chunk per 1024 / 256 / 128 /
// 64 buckets 13.65 / 9.86 / 9.20 / 9.91 ms, no failures or false negatives.
#ifndef PG_BATCH_INSERT_BUCKETS
#define PG_BATCH_INSERT_BUCKETS 128
#endif
constexpr uint64_t kBatchMaxChunk = 16384;
__device__ __forceinline__ uint64_t batch_chunk_keys(const batch_args &a, const pg_op_desc &od)
{
    if (PG_BATCH_INSERT_BUCKETS == 0 || (od.op != PG_OP_INSERT && od.op != PG_OP_INSERT_WITH_DELETE) ||
        od.table >= a.ntables)
        return kBatchChunk;
    const uint64_t nb = a.tables[od.table].lv[0].nbmod.d;
    const uint64_t chunks = nb >= PG_BATCH_INSERT_BUCKETS ? nb / PG_BATCH_INSERT_BUCKETS : 1;
    const uint64_t per = (od.count + chunks - 1) / chunks;
    // a request far larger than its table (mostly failing inserts) still
    // spreads over warps: at most kBatchMaxChunk keys per chunk
    return per > kBatchChunk ? (per < kBatchMaxChunk ? per : kBatchMaxChunk) : kBatchChunk;
}

// one block: exclusive scan of ceil(count / batch_chunk_keys) over the requests
__global__ void __launch_bounds__(1024) k_batch_plan(batch_args a);

template <int FMT, int B, int G, int S0, bool BK>
__global__ void __launch_bounds__(256, min_blocks_of<FMT, G>()) k_batch(batch_args a)
{
    using F = fmt_t<FMT>;
    using V = typename F::V;
    using T = table_ops<FMT, B, G, S0, BK>;
    const group<G> g = group<G>::make();
    const uint32_t lane = threadIdx.x & 31u;
    constexpr uint32_t kGroupsPerWarp = 32 / G;
    const uint32_t gi = lane / G;  // group index inside the warp
    uint32_t nops = *a.nops;
    if (nops > a.max_ops) nops = a.max_ops;
    const unsigned long long total = a.chunk_start[nops];
    const V *vin = static_cast<const V *>(a.vals_in);
    V *vout = static_cast<V *>(a.vals_out);
    while (true) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(a.work, 1ULL);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= total) break;
        // the request whose chunks contain c: last j with chunk_start[j] <= c
        uint32_t lo = 0, hi = nops;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (a.chunk_start[mid] <= c) lo = mid;
            else hi = mid;
        }
        const pg_op_desc od = a.ops[lo];
        if (od.table >= a.ntables || od.op > PG_OP_REMOVE) continue;  // malformed request: skipped
        const table_desc &t = a.tables[od.table];
        const uint64_t ck = batch_chunk_keys(a, od);
        const uint64_t first = od.offset + (c - a.chunk_start[lo]) * ck;
        const uint64_t end = od.offset + od.count;
        const uint64_t stop = first + ck < end ? first + ck : end;
        uint32_t cnt = 0;
        for (uint64_t i = first + gi; i < stop; i += kGroupsPerWarp) {
            const uint64_t key = __ldg(a.keys + i);
            bool r;
            if (od.op == PG_OP_INSERT) {
                r = T::insert(t, g, key, vin ? __ldg(vin + i) : (V)0);
                if (g.gl == 0) cnt += !r;
            } else if (od.op == PG_OP_QUERY) {
                V v = 0;
                r = T::query(t, g, key, v);
                if (g.gl == 0) {
                    if (vout) __stcs(vout + i, r ? v : (V)0);
                    cnt += r;
                }
            } else {
                r = T::remove(t, g, key);
                if (g.gl == 0) cnt += r;
            }
            if (g.gl == 0 && a.flags) __stcs(a.flags + i, (uint8_t)r);
        }
        if (a.op_counts) {
            cnt = __reduce_add_sync(0xffffffffu, cnt);
            if (lane == 0 && cnt) atomicAdd(a.op_counts + lo, (unsigned long long)cnt);
        }
    }
}

template <int FMT, int B, int G>
cudaError_t batch_bg(const batch_args &a, int scheme, bool bk, dim3 grid, dim3 block, cudaStream_t s)
{
    if (scheme == SCHEME_BUCKET) {
        if (bk) k_batch<FMT, B, G, SCHEME_BUCKET, true><<<grid, block, 0, s>>>(a);
        else k_batch<FMT, B, G, SCHEME_BUCKET, false><<<grid, block, 0, s>>>(a);
    } else {
        if (bk) k_batch<FMT, B, G, SCHEME_TWO_CHOICE, true><<<grid, block, 0, s>>>(a);
        else k_batch<FMT, B, G, SCHEME_TWO_CHOICE, false><<<grid, block, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <int FMT, int B>
cudaError_t batch_b(const batch_args &a, uint32_t lanes, int scheme, bool bk, dim3 grid, dim3 block, cudaStream_t s)
{
    switch (lanes) {
    case 1: return batch_bg<FMT, B, 1>(a, scheme, bk, grid, block, s);
    case 2: return batch_bg<FMT, B, 2>(a, scheme, bk, grid, block, s);
    case 4: return batch_bg<FMT, B, 4>(a, scheme, bk, grid, block, s);
    case 8:
        if constexpr (B >= 8) return batch_bg<FMT, B, 8>(a, scheme, bk, grid, block, s);
        else return cudaErrorInvalidConfiguration;
    case 16:
        if constexpr (B >= 16) return batch_bg<FMT, B, 16>(a, scheme, bk, grid, block, s);
        else return cudaErrorInvalidConfiguration;
    default: return cudaErrorInvalidConfiguration;
    }
}

template <int FMT>
cudaError_t batch_fmt(const batch_args &a, uint32_t bucket, uint32_t lanes, int scheme, bool bk, dim3 grid,
                      dim3 block, cudaStream_t s)
{
    switch (bucket) {
    case 4: return batch_b<FMT, 4>(a, lanes, scheme, bk, grid, block, s);
    case 8: return batch_b<FMT, 8>(a, lanes, scheme, bk, grid, block, s);
    case 16: return batch_b<FMT, 16>(a, lanes, scheme, bk, grid, block, s);
    case 32: return batch_b<FMT, 32>(a, lanes, scheme, bk, grid, block, s);
    default: return cudaErrorInvalidConfiguration;
    }
}

#define PG_DECLARE_BATCH(name)                                                                                   \
    cudaError_t name(const batch_args &a, uint32_t bucket, uint32_t lanes, int scheme, bool bk, dim3 grid, \
                     dim3 block, cudaStream_t s)
PG_DECLARE_BATCH(batch_kv64);
PG_DECLARE_BATCH(batch_kv64_split);
PG_DECLARE_BATCH(batch_tagval16);
PG_DECLARE_BATCH(batch_tagval16_split);
PG_DECLARE_BATCH(batch_tag16);
PG_DECLARE_BATCH(batch_kv64_fp);
// the bucketed filter: level-0 bucket b0, backing bucket b1 (packed formats)
cudaError_t batch_packed(const batch_args &a, uint32_t ifmt, uint32_t b0, uint32_t b1, uint32_t lanes, bool bk,
                         dim3 grid, dim3 block, cudaStream_t s);

}  // namespace pg
