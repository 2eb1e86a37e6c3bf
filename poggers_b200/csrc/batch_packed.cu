// batch_packed.cu -- multi-table batch kernels for the bucketed filter
// (packed (tag, value) slots; see include/poggers_b200/packed.cuh).  Same
// plan and chunk claiming as k_batch; the per-key work is the bulk packed
// kernels' (packed_table::op), with PG_OP_INSERT_WITH_DELETE besides insert,
// query and remove.
#include "batch_kernels.cuh"
#include "bulk_packed.cuh"

namespace pg {

template <int W, int B0, int B1, int G, bool BK>
__global__ void __launch_bounds__(256) k_batch_packed(batch_args a)
{
    using T = packed_table<W, B0, B1, G, BK>;
    using V = typename pk<W>::V;
    const group<G> g = group<G>::make();
    const uint32_t lane = threadIdx.x & 31u;
    constexpr uint32_t kGroupsPerWarp = 32 / G;
    const uint32_t gi = lane / G;
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
        uint32_t lo = 0, hi = nops;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (a.chunk_start[mid] <= c) lo = mid;
            else hi = mid;
        }
        const pg_op_desc od = a.ops[lo];
        if (od.table >= a.ntables || od.op > PG_OP_INSERT_WITH_DELETE) continue;  // malformed request: skipped
        const table_desc &t = a.tables[od.table];
        const int opk = od.op == PG_OP_INSERT      ? (int)POP_INSERT
                        : od.op == PG_OP_QUERY     ? (int)POP_QUERY
                        : od.op == PG_OP_REMOVE    ? (int)POP_REMOVE
                                                   : (int)POP_INSERT_DELETE;
        const bool counts_hits = opk == POP_QUERY || opk == POP_REMOVE;
        const uint64_t ck = batch_chunk_keys(a, od);
        const uint64_t first = od.offset + (c - a.chunk_start[lo]) * ck;
        const uint64_t end = od.offset + od.count;
        const uint64_t stop = first + ck < end ? first + ck : end;
        uint32_t cnt = 0;
        for (uint64_t i = first + gi; i < stop; i += kGroupsPerWarp) {
            const uint64_t key = __ldg(a.keys + i);
            const uint64_t val = (vin && (opk == POP_INSERT || opk == POP_INSERT_DELETE)) ? (uint64_t)__ldg(vin + i) : 0;
            V out = 0;
            bool found = false;
            const bool r = T::op(t, g, opk, key, val, out, found);
            if (g.gl == 0) {
                if (opk == POP_QUERY && vout) vout[i] = r ? out : (V)0;
                if (a.flags) a.flags[i] = (uint8_t)r;
                cnt += counts_hits ? (uint32_t)r : (uint32_t)!r;
            }
        }
        if (a.op_counts) {
            cnt = __reduce_add_sync(0xffffffffu, cnt);
            if (lane == 0 && cnt) atomicAdd(a.op_counts + lo, (unsigned long long)cnt);
        }
    }
}

template <int W, int B0, int G>
cudaError_t batch_packed_b0(const batch_args &a, uint32_t b1, bool bk, dim3 grid, dim3 block, cudaStream_t s)
{
    if (!bk) k_batch_packed<W, B0, 8, G, false><<<grid, block, 0, s>>>(a);
    else if (b1 == 8) k_batch_packed<W, B0, 8, G, true><<<grid, block, 0, s>>>(a);
    else if (b1 == 16) k_batch_packed<W, B0, 16, G, true><<<grid, block, 0, s>>>(a);
    else return cudaErrorInvalidConfiguration;
    return cudaGetLastError();
}

template <int W>
cudaError_t batch_packed_w(const batch_args &a, uint32_t b0, uint32_t b1, uint32_t lanes, bool bk, dim3 grid,
                           dim3 block, cudaStream_t s)
{
    const bool four = lanes >= 4;
    switch (b0) {
    case 8: return four ? batch_packed_b0<W, 8, 4>(a, b1, bk, grid, block, s) : batch_packed_b0<W, 8, 1>(a, b1, bk, grid, block, s);
    case 16: return four ? batch_packed_b0<W, 16, 4>(a, b1, bk, grid, block, s) : batch_packed_b0<W, 16, 1>(a, b1, bk, grid, block, s);
    case 32: return four ? batch_packed_b0<W, 32, 4>(a, b1, bk, grid, block, s) : batch_packed_b0<W, 32, 1>(a, b1, bk, grid, block, s);
    default: return cudaErrorInvalidConfiguration;
    }
}

cudaError_t batch_packed(const batch_args &a, uint32_t ifmt, uint32_t b0, uint32_t b1, uint32_t lanes, bool bk,
                         dim3 grid, dim3 block, cudaStream_t s)
{
    return ifmt == FMT_PACKED16 ? batch_packed_w<16>(a, b0, b1, lanes, bk, grid, block, s)
                                : batch_packed_w<8>(a, b0, b1, lanes, bk, grid, block, s);
}

}  // namespace pg
