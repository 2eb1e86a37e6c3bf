// diag.cu -- random-access ceilings of the GPU (no counterpart in the
// reference).
//
// The filters' kernels touch one or two 32-byte DRAM sectors at random
// addresses per key, and claim slots with an atomic on a sector they have just
// read.  Their bound is therefore the rate at which the memory system serves
// random sectors and random read-modify-writes, not the streaming copy
// bandwidth.  These kernels measure those rates with nothing else in the way:
// every thread issues several independent accesses at once (addresses from a
// hash of the access index, so no index array is read), and the results only
// feed a checksum.
#include <stdint.h>
#include <cuda_runtime.h>

#include "poggers_b200.h"

namespace {

constexpr int kUnroll = 4;  // independent accesses in flight per thread

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    // splitmix64's finaliser (Steele, Lea and Flood 2014)
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ void ld_sector(const unsigned char *p, unsigned long long (&v)[4])
{
    asm volatile("ld.global.cg.v4.u64 {%0, %1, %2, %3}, [%4];"
                 : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3])
                 : "l"(p));
}

// MODE: PG_DIAG_READ32, PG_DIAG_READ64, PG_DIAG_READ32_CAS, PG_DIAG_RED32,
// PG_DIAG_READ32_CAS_NEXT.  Unit = the aligned span one access picks at
// random: 32 B, 64 B, 32 B, 4 B, 64 B.
// Every offset is mulhi(hash, units) * unit < units * unit <= the buffer's bytes.
template <int MODE>
__global__ void __launch_bounds__(256) k_random_access(unsigned char *buf, uint64_t units, uint64_t per_thread,
                                                       uint64_t seed, unsigned long long *sink)
{
    constexpr uint64_t kUnit =
        (MODE == PG_DIAG_READ64 || MODE == PG_DIAG_READ32_CAS_NEXT) ? 64 : (MODE == PG_DIAG_RED32 ? 4 : 32);
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long acc = 0;
    for (uint64_t j = 0; j < per_thread; j += kUnroll) {
        uint64_t off[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) off[u] = __umul64hi(mix64(seed + tid * per_thread + j + u), units) * kUnit;
        if constexpr (MODE == PG_DIAG_RED32) {
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) atomicAdd(reinterpret_cast<unsigned *>(buf + off[u]), 1u);
        } else {
            unsigned long long v[kUnroll][4];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) ld_sector(buf + off[u], v[u]);
            if constexpr (MODE == PG_DIAG_READ64) {
                unsigned long long w[kUnroll][4];
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) ld_sector(buf + off[u] + 32, w[u]);
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) acc ^= w[u][0] ^ w[u][3];
            }
            if constexpr (MODE == PG_DIAG_READ32_CAS || MODE == PG_DIAG_READ32_CAS_NEXT) {
                // claim the sector's first word: a CAS on the value just read
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    const unsigned seen = (unsigned)v[u][0];
                    acc ^= atomicCAS(reinterpret_cast<unsigned *>(buf + off[u]), seen, seen + 1u);
                }
            }
            if constexpr (MODE == PG_DIAG_READ32_CAS_NEXT) {
                // then the value: 2 bytes of the span's second sector
#pragma unroll
                for (int u = 0; u < kUnroll; ++u)
                    *reinterpret_cast<unsigned short *>(buf + off[u] + 32 + 2 * (u & 15)) = (unsigned short)v[u][1];
            }
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) acc ^= v[u][0] ^ v[u][1] ^ v[u][2] ^ v[u][3];
        }
    }
    if (acc == 0x9E3779B97F4A7C15ull) atomicXor(sink, acc);  // keeps the loads; practically never taken
}

}  // namespace

extern "C" {

pg_status pg_diag_random_access(void *d_buf, uint64_t bytes, uint32_t mode, uint64_t accesses, uint64_t seed,
                                uint32_t blocks_per_sm, uint64_t *accesses_done, uint64_t *d_sink,
                                pg_stream_t stream)
{
    if (!d_buf || !d_sink || mode > PG_DIAG_READ32_CAS_NEXT || bytes < 64 || ((uintptr_t)d_buf & 63))
        return PG_ERR_INVALID;
    if (blocks_per_sm == 0) blocks_per_sm = 8;
    if (blocks_per_sm > 8) return PG_ERR_INVALID;  // 8 x 256 threads fill an SM
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return PG_ERR_CUDA;
    }
    const uint64_t unit =
        (mode == PG_DIAG_READ64 || mode == PG_DIAG_READ32_CAS_NEXT) ? 64 : (mode == PG_DIAG_RED32 ? 4 : 32);
    const uint64_t units = bytes / unit;
    const uint64_t threads = (uint64_t)sms * blocks_per_sm * 256;
    uint64_t per_thread = (accesses + threads - 1) / threads;
    per_thread = (per_thread + kUnroll - 1) / kUnroll * kUnroll;
    if (per_thread == 0) per_thread = kUnroll;
    if (accesses_done) *accesses_done = per_thread * threads;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned char *b = static_cast<unsigned char *>(d_buf);
    unsigned long long *sk = reinterpret_cast<unsigned long long *>(d_sink);
    const dim3 grid((unsigned)(sms * blocks_per_sm)), block(256);
    switch (mode) {
    case PG_DIAG_READ32: k_random_access<PG_DIAG_READ32><<<grid, block, 0, s>>>(b, units, per_thread, seed, sk); break;
    case PG_DIAG_READ64: k_random_access<PG_DIAG_READ64><<<grid, block, 0, s>>>(b, units, per_thread, seed, sk); break;
    case PG_DIAG_READ32_CAS:
        k_random_access<PG_DIAG_READ32_CAS><<<grid, block, 0, s>>>(b, units, per_thread, seed, sk);
        break;
    case PG_DIAG_READ32_CAS_NEXT:
        k_random_access<PG_DIAG_READ32_CAS_NEXT><<<grid, block, 0, s>>>(b, units, per_thread, seed, sk);
        break;
    default: k_random_access<PG_DIAG_RED32><<<grid, block, 0, s>>>(b, units, per_thread, seed, sk); break;
    }
    return cudaGetLastError() == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

}  // extern "C"
