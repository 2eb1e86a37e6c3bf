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

// Resident blocks of 256 the register allocation must allow.  Held to 6
// (40 registers, a few words spilled) the kernels keep 1.5x the keys in flight
// of their natural 62-64 registers (4 blocks); measured on the delete flow
// (insert, remove, query, re-add):
//   4 lanes: held 1.33x and 1.35x faster at 2^24 and 2^28 slots;
//   1 lane:  held 1.10x, 1.14x, 1.05x faster at 2^24, 2^25, 2^26 slots (64 to
//            256 MiB, much of it in L2), 0.93x at 2^27 and 2^28 (0.5 and
//            1 GiB: random DRAM sector reads bound them, and the spilled
//            words only add traffic).
// So the one-lane kernels are built both ways and chosen per launch by the
// primary level's bytes.
constexpr int kPackedHeldBlocks = 6;
#ifndef PG_PACKED_HELD_MAX_MB
#define PG_PACKED_HELD_MAX_MB 256
#endif
constexpr uint64_t kPackedHeldMaxBytes = (uint64_t)PG_PACKED_HELD_MAX_MB << 20;

template <int W, int B0, int B1, int G, bool BK, int OP, int MINB>
__global__ void __launch_bounds__(256, MINB) k_bulk_packed(table_desc t, packed_args a)
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

template <int W, int B0, int B1, int G, bool BK, int MINB>
cudaError_t launch_packed_minb(int op, const table_desc &t, const packed_args &a, dim3 grid, dim3 block,
                               cudaStream_t s)
{
    switch (op) {
    case POP_INSERT: k_bulk_packed<W, B0, B1, G, BK, POP_INSERT, MINB><<<grid, block, 0, s>>>(t, a); break;
    case POP_QUERY: k_bulk_packed<W, B0, B1, G, BK, POP_QUERY, MINB><<<grid, block, 0, s>>>(t, a); break;
    case POP_REMOVE: k_bulk_packed<W, B0, B1, G, BK, POP_REMOVE, MINB><<<grid, block, 0, s>>>(t, a); break;
    case POP_INSERT_DELETE: k_bulk_packed<W, B0, B1, G, BK, POP_INSERT_DELETE, MINB><<<grid, block, 0, s>>>(t, a); break;
    case POP_INSERT_IF_NOT_EXISTS:
        k_bulk_packed<W, B0, B1, G, BK, POP_INSERT_IF_NOT_EXISTS, MINB><<<grid, block, 0, s>>>(t, a);
        break;
    default: k_bulk_packed<W, B0, B1, G, BK, POP_INSERT_IF_NOT_EXISTS_DELETE, MINB><<<grid, block, 0, s>>>(t, a); break;
    }
    return cudaGetLastError();
}

template <int W, int B0, int B1, int G, bool BK>
cudaError_t launch_packed_op(int op, const table_desc &t, const packed_args &a, dim3 grid, dim3 block,
                             cudaStream_t s)
{
    if constexpr (G > 1) {
        return launch_packed_minb<W, B0, B1, G, BK, kPackedHeldBlocks>(op, t, a, grid, block, s);
    } else {
        const uint64_t bytes = t.lv[0].nbmod.d * (uint64_t)t.lv[0].bucket_bytes;
        if (bytes <= kPackedHeldMaxBytes)
            return launch_packed_minb<W, B0, B1, G, BK, kPackedHeldBlocks>(op, t, a, grid, block, s);
        return launch_packed_minb<W, B0, B1, G, BK, 1>(op, t, a, grid, block, s);
    }
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
