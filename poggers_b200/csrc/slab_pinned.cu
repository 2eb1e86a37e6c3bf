// slab_pinned.cu -- C ABI of the pinned slab pool: the reference's slab policy
// (per-SM pinned slabs with backups, whole-word claims with a per-SM cache,
// pivot and pool) behind pg_pslab_*; the template API's
// one_size_slab_allocator<extra_blocks> is built on it.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime.h>

#include <vector>

#include "poggers_b200.h"
#include "on_device.h"
#include "poggers_b200/slab_pinned.cuh"

using namespace pg;

struct pg_pslab {
    pslab_desc d;
    uint64_t pool_bytes;
    int device;
};

namespace {

pg_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return PG_OK;
    if (e == cudaErrorMemoryAllocation) return PG_ERR_NOMEM;
    return PG_ERR_CUDA;
}

__global__ void k_pslab_nsmid(unsigned *out)
{
    unsigned n;
    asm volatile("mov.u32 %0, %%nsmid;" : "=r"(n));
    *out = n;
}

// Everything empty and in the pool, then every SM id pins a primary and E
// backups, SMs in order (init_with_allocators_memory, offset_slab.cuh:1710-1748):
// SM m's place i takes slab m * (E + 1) + i while slabs last.
__global__ void k_pslab_init(pslab_desc S)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t per = (uint64_t)S.extra + 1;
    const uint64_t pinned = S.nslabs < per * S.nsm ? S.nslabs : per * S.nsm;
    for (uint64_t i = tid; i < S.nslabs * 64; i += stride) S.bits[i] = ~0ULL;
    for (uint64_t s = tid; s < S.nslabs; s += stride) {
        S.mgr[s] = ~0ULL;
        S.pinned[s] = s < pinned ? 1u : 0u;
    }
    const uint64_t nw = (S.nslabs + 63) / 64;
    for (uint64_t w = tid; w < nw; w += stride) {
        unsigned long long m = 0;
        for (uint64_t b = 0; b < 64; ++b) {
            const uint64_t s = w * 64 + b;
            if (s < S.nslabs && s >= pinned) m |= 1ULL << b;
        }
        S.in_pool[w] = m;
    }
    for (uint64_t i = tid; i < (uint64_t)S.nsm * kPinnedPlaces; i += stride) {
        const uint64_t m = i / kPinnedPlaces, p = i % kPinnedPlaces;
        const uint64_t s = m * per + p;
        S.pin[i] = (p < per && s < pinned) ? (long long)s : -1LL;
        S.cache_bits[i] = 0;
        S.cache_base[i] = 0;
    }
    for (uint64_t m = tid; m < S.nsm; m += stride) {
        unsigned long long mk = 0;
        for (uint64_t p = 0; p < per; ++p)
            if (m * per + p < pinned) mk |= 1ULL << p;
        S.markers[m] = mk;
        S.cache_claim[m] = ~0ULL;
        S.cache_mgr[m] = 0;
    }
    if (tid < 3) S.stats[tid] = 0;
}

__global__ void __launch_bounds__(256) k_pslab_malloc(pslab_desc S, uint64_t n, void **out, unsigned long long *fails)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    void *p = pslab_malloc(S);
    out[i] = p;
    if (!p && fails) atomicAdd(fails, 1ULL);
}

// one warp, `rounds` malloc() calls of `group` lanes each, in order
__global__ void k_pslab_serial_malloc(pslab_desc S, uint32_t rounds, uint32_t group, void **out,
                                      unsigned long long *fails)
{
    if (threadIdx.x >= group) return;
    const unsigned m = group == 32 ? 0xffffffffu : ((1u << group) - 1u);
    for (uint32_t k = 0; k < rounds; ++k) {
        __syncwarp(m);
        void *p = pslab_malloc(S);
        out[(uint64_t)k * group + threadIdx.x] = p;
        if (!p && fails) atomicAdd(fails, 1ULL);
    }
}

// counts[0..3]: refused, freed, returned to the pool, emptied while pinned
__global__ void __launch_bounds__(256) k_pslab_free(pslab_desc S, uint64_t n, void *const *ptrs,
                                                    unsigned long long *counts, uint32_t serial)
{
    if (serial) {
        if (blockIdx.x || threadIdx.x) return;
        for (uint64_t i = 0; i < n; ++i)
            if (ptrs[i]) atomicAdd(counts + pslab_release(S, ptrs[i]), 1ULL);
        return;
    }
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (ptrs[i]) atomicAdd(counts + pslab_release(S, ptrs[i]), 1ULL);
}

unsigned grid_for(uint64_t n)
{
    uint64_t b = (n + 255) / 256;
    return (unsigned)(b ? b : 1);
}

}  // namespace

extern "C" {

pg_status pg_pslab_create(uint64_t num_allocs, uint64_t object_bytes, uint32_t extra_blocks, pg_pslab **out)
{
    if (!out || num_allocs == 0 || object_bytes == 0 || extra_blocks + 1 >= kPinnedPlaces) return PG_ERR_INVALID;
    *out = nullptr;
    const uint64_t nslabs = (num_allocs - 1) / kPinnedObjects + 1;  // slab_one_size.cuh:94
    if (nslabs > 0xFFFFFFFEull || object_bytes > ~0ull / (nslabs * kPinnedObjects)) return PG_ERR_INVALID;
    pg_pslab *a = (pg_pslab *)calloc(1, sizeof(pg_pslab));
    if (!a) return PG_ERR_NOMEM;
    if (cudaGetDevice(&a->device) != cudaSuccess) {
        cudaGetLastError();
        free(a);
        return PG_ERR_CUDA;
    }
    a->d.nslabs = nslabs;
    a->d.size = object_bytes;
    a->d.extra = extra_blocks;
    a->pool_bytes = nslabs * kPinnedObjects * object_bytes;
    unsigned *d_n = nullptr, nsm = 0;
    cudaError_t e = cudaMalloc(&d_n, 4);
    if (e == cudaSuccess) {
        k_pslab_nsmid<<<1, 1>>>(d_n);
        e = cudaMemcpy(&nsm, d_n, 4, cudaMemcpyDeviceToHost);
        cudaFree(d_n);
    }
    if (e == cudaSuccess && nsm == 0) e = cudaErrorUnknown;
    a->d.nsm = nsm;
    const uint64_t nw = (nslabs + 63) / 64, places = (uint64_t)nsm * kPinnedPlaces;
    if (e == cudaSuccess) e = cudaMalloc(&a->d.pool, a->pool_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.mgr, nslabs * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.bits, nslabs * 64 * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.pinned, nslabs * 4);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.in_pool, nw * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.cache_claim, (uint64_t)nsm * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.cache_mgr, (uint64_t)nsm * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.cache_bits, places * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.cache_base, places * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.pin, places * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.markers, (uint64_t)nsm * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.stats, 3 * 8);
    if (e == cudaSuccess) {
        k_pslab_init<<<grid_for(nslabs * 64 < 4096 * 256 ? nslabs * 64 : 4096 * 256), 256>>>(a->d);
        e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        pg_pslab_destroy(a);
        return cuda_status(e);
    }
    *out = a;
    return PG_OK;
}

pg_status pg_pslab_destroy(pg_pslab *a)
{
    if (!a) return PG_ERR_INVALID;
    cudaFree(a->d.pool);
    cudaFree(a->d.mgr);
    cudaFree(a->d.bits);
    cudaFree(a->d.pinned);
    cudaFree(a->d.in_pool);
    cudaFree(a->d.cache_claim);
    cudaFree(a->d.cache_mgr);
    cudaFree(a->d.cache_bits);
    cudaFree(a->d.cache_base);
    cudaFree(a->d.pin);
    cudaFree(a->d.markers);
    cudaFree(a->d.stats);
    free(a);
    return PG_OK;
}

pg_status pg_pslab_desc(const pg_pslab *a, void *out_desc, uint64_t bytes)
{
    if (!a || !out_desc || bytes != sizeof(pslab_desc)) return PG_ERR_INVALID;
    memcpy(out_desc, &a->d, sizeof(pslab_desc));
    return PG_OK;
}

pg_status pg_pslab_report(const pg_pslab *a, uint64_t *pool_slabs, uint64_t *max_slabs, uint64_t *sm_ids,
                          uint64_t *double_frees)
{
    if (!a || !pg_on_device(a->device)) return PG_ERR_INVALID;
    const uint64_t nw = (a->d.nslabs + 63) / 64;
    std::vector<unsigned long long> h(nw);
    unsigned long long st[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpy(h.data(), a->d.in_pool, nw * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(st, a->d.stats, sizeof(st), cudaMemcpyDeviceToHost);
    uint64_t n = 0;
    for (unsigned long long w : h) n += (uint64_t)__builtin_popcountll(w);
    if (pool_slabs) *pool_slabs = n;
    if (max_slabs) *max_slabs = a->d.nslabs;
    if (sm_ids) *sm_ids = a->d.nsm;
    if (double_frees) *double_frees = st[0];
    return cuda_status(e);
}

pg_status pg_pslab_bulk_malloc(pg_pslab *a, uint64_t n, void **d_ptrs, uint64_t *d_fail_count, pg_stream_t stream)
{
    if (!a || (n && !d_ptrs) || !pg_on_device(a->device)) return PG_ERR_INVALID;
    if (n == 0) return PG_OK;
    k_pslab_malloc<<<grid_for(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        a->d, n, d_ptrs, reinterpret_cast<unsigned long long *>(d_fail_count));
    return cuda_status(cudaGetLastError());
}

pg_status pg_pslab_serial_malloc(pg_pslab *a, uint32_t rounds, uint32_t group, void **d_ptrs, uint64_t *d_fail_count,
                                 pg_stream_t stream)
{
    if (!a || !d_ptrs || group == 0 || group > 32 || !pg_on_device(a->device)) return PG_ERR_INVALID;
    if (rounds == 0) return PG_OK;
    k_pslab_serial_malloc<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        a->d, rounds, group, d_ptrs, reinterpret_cast<unsigned long long *>(d_fail_count));
    return cuda_status(cudaGetLastError());
}

pg_status pg_pslab_bulk_free(pg_pslab *a, void *const *d_ptrs, uint64_t n, uint64_t *d_counts, int serial,
                             pg_stream_t stream)
{
    if (!a || !d_counts || (n && !d_ptrs) || !pg_on_device(a->device)) return PG_ERR_INVALID;
    if (n == 0) return PG_OK;
    unsigned blocks = serial ? 1u : grid_for(n);
    if (blocks > a->d.nsm * 32u) blocks = a->d.nsm * 32u;  // grid-stride; %nsmid >= the SM count
    k_pslab_free<<<blocks, serial ? 32 : 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        a->d, n, d_ptrs, reinterpret_cast<unsigned long long *>(d_counts), serial ? 1u : 0u);
    return cuda_status(cudaGetLastError());
}

}  // extern "C"
