// bulk_packed.cuh -- bulk kernels of the bucketed filter with tombstone reuse
// (packed (tag, value) slots; see include/poggers_b200/packed.cuh).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "poggers_b200/packed.cuh"
#include "bulk_kernels.cuh"

namespace pg {

struct packed_args {
    const uint64_t *keys;
    const void *vals_in;            // V per key (uint16 for 16-bit tags, uint8 for 8-bit), or null = 0
    void *vals_out;                 // V per key: the value found (query, insert_if_not_exists*)
    uint8_t *flags;                 // the operation's boolean per key
    uint8_t *found;                 // insert_if_not_exists*: the key was already present
    unsigned long long *count;      // query / remove: successes; insert forms: failures
    uint64_t n;
};

// build knob: resident blocks the register allocation must allow; 1 measured
// fastest on the delete flow at 2^28 slots (5: -3.5 %, 6: -7 %, from spills)
#ifndef PG_PACKED_MIN_BLOCKS
#define PG_PACKED_MIN_BLOCKS 1
#endif

template <int W, int B0, int B1, int G, bool BK, int OP>
__global__ void __launch_bounds__(256, PG_PACKED_MIN_BLOCKS) k_bulk_packed(table_desc t, packed_args a)
{
    using T = packed_table<W, B0, B1, G, BK>;
    using V = typename pk<W>::V;
    const group<G> g = group<G>::make();
    const uint64_t gid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
    const V *vin = static_cast<const V *>(a.vals_in);
    V *vout = static_cast<V *>(a.vals_out);
    uint32_t c = 0;
    for (uint64_t i = gid; i < a.n; i += ngroups) {
        const uint64_t key = __ldg(a.keys + i);
        const uint64_t val = vin ? (uint64_t)__ldg(vin + i) : 0;
        V out = 0;
        bool found = false;
        const bool r = T::op(t, g, OP, key, val, out, found);
        if (g.gl == 0) {
            if (a.flags) a.flags[i] = (uint8_t)r;
            if constexpr (OP == POP_QUERY || OP == POP_INSERT_IF_NOT_EXISTS || OP == POP_INSERT_IF_NOT_EXISTS_DELETE)
                if (vout) vout[i] = r ? out : (V)0;
            if constexpr (OP == POP_INSERT_IF_NOT_EXISTS || OP == POP_INSERT_IF_NOT_EXISTS_DELETE)
                if (a.found) a.found[i] = (uint8_t)found;
            c += (OP == POP_QUERY || OP == POP_REMOVE) ? (uint32_t)r : (uint32_t)!r;
        }
    }
    add_count(a.count, c);
}

template <int W, int B0, int B1, int G, bool BK>
cudaError_t launch_packed_op(int op, const table_desc &t, const packed_args &a, dim3 grid, dim3 block,
                             cudaStream_t s)
{
    switch (op) {
    case POP_INSERT: k_bulk_packed<W, B0, B1, G, BK, POP_INSERT><<<grid, block, 0, s>>>(t, a); break;
    case POP_QUERY: k_bulk_packed<W, B0, B1, G, BK, POP_QUERY><<<grid, block, 0, s>>>(t, a); break;
    case POP_REMOVE: k_bulk_packed<W, B0, B1, G, BK, POP_REMOVE><<<grid, block, 0, s>>>(t, a); break;
    case POP_INSERT_DELETE: k_bulk_packed<W, B0, B1, G, BK, POP_INSERT_DELETE><<<grid, block, 0, s>>>(t, a); break;
    case POP_INSERT_IF_NOT_EXISTS:
        k_bulk_packed<W, B0, B1, G, BK, POP_INSERT_IF_NOT_EXISTS><<<grid, block, 0, s>>>(t, a);
        break;
    default: k_bulk_packed<W, B0, B1, G, BK, POP_INSERT_IF_NOT_EXISTS_DELETE><<<grid, block, 0, s>>>(t, a); break;
    }
    return cudaGetLastError();
}

// backing bucket: 8 or 16 slots (the reference's backing tables use 8)
template <int W, int B0, int G>
cudaError_t launch_packed_b0(int op, uint32_t b1, const table_desc &t, const packed_args &a, dim3 grid, dim3 block,
                             cudaStream_t s)
{
    if (t.nlevels < 2) return launch_packed_op<W, B0, 8, G, false>(op, t, a, grid, block, s);
    if (b1 == 8) return launch_packed_op<W, B0, 8, G, true>(op, t, a, grid, block, s);
    if (b1 == 16) return launch_packed_op<W, B0, 16, G, true>(op, t, a, grid, block, s);
    return cudaErrorInvalidConfiguration;
}

// lanes per key: 1 or 4 (a launch knob; results do not depend on it)
template <int W>
cudaError_t launch_packed(int op, uint32_t b0, uint32_t b1, uint32_t lanes, const table_desc &t,
                          const packed_args &a, dim3 grid, dim3 block, cudaStream_t s)
{
    const bool four = lanes >= 4;
    switch (b0) {
    case 8: return four ? launch_packed_b0<W, 8, 4>(op, b1, t, a, grid, block, s)
                        : launch_packed_b0<W, 8, 1>(op, b1, t, a, grid, block, s);
    case 16: return four ? launch_packed_b0<W, 16, 4>(op, b1, t, a, grid, block, s)
                         : launch_packed_b0<W, 16, 1>(op, b1, t, a, grid, block, s);
    case 32: return four ? launch_packed_b0<W, 32, 4>(op, b1, t, a, grid, block, s)
                         : launch_packed_b0<W, 32, 1>(op, b1, t, a, grid, block, s);
    default: return cudaErrorInvalidConfiguration;
    }
}

cudaError_t launch_packed16(int op, uint32_t b0, uint32_t b1, uint32_t lanes, const table_desc &t,
                            const packed_args &a, dim3 grid, dim3 block, cudaStream_t s);
cudaError_t launch_packed8(int op, uint32_t b0, uint32_t b1, uint32_t lanes, const table_desc &t,
                           const packed_args &a, dim3 grid, dim3 block, cudaStream_t s);

}  // namespace pg
