// slab.cu -- C ABI of the slab allocator: pools, bulk malloc / free, fill reports.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime.h>
#include <vector>

#include "poggers_b200.h"
#include "on_device.h"
#include "poggers_b200/slab.cuh"

using namespace pg;

struct pg_slab {
    slab_desc d;
    uint64_t capacity;
    uint64_t pool_bytes;
    int device;
    int num_sms;
};

struct pg_slab_set {
    uint32_t nclasses;
    pg_slab *cls[PG_SLAB_MAX_CLASSES];
    uint64_t class_bytes[PG_SLAB_MAX_CLASSES];
};

namespace {

pg_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return PG_OK;
    if (e == cudaErrorMemoryAllocation) return PG_ERR_NOMEM;
    return PG_ERR_CUDA;
}

__global__ void k_slab_init(slab_desc S)
{
    const uint64_t words = S.nslabs * kSlabWords;
    const uint64_t nsum = (S.nslabs + 63) / 64;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x) {
        S.bits[i] = ~0ULL;
        if (i < S.nslabs) S.mgr[i] = ~0ULL;
        if (i < nsum) {
            const uint64_t left = S.nslabs - i * 64;
            S.summary[i] = left >= 64 ? ~0ULL : ((1ULL << left) - 1);
        }
        if (i < kSlabCursors) S.cursor[i] = (uint32_t)((i * S.nslabs) / kSlabCursors);
        if (i < 2) S.stats[i] = 0;
    }
}

__global__ void __launch_bounds__(256) k_slab_malloc(slab_desc S, uint64_t n, void **out, unsigned long long *fails)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    void *p = slab_malloc(S);
    out[i] = p;
    if (!p && fails) atomicAdd(fails, 1ULL);
}

__global__ void __launch_bounds__(256) k_slab_free(slab_desc S, uint64_t n, void *const *ptrs, unsigned long long *bad)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const void *p = ptrs[i];
        if (!p) continue;  // free(nullptr) is a no-op
        if (!slab_release(S, p) && bad) atomicAdd(bad, 1ULL);
    }
}

__global__ void __launch_bounds__(256) k_slab_count(slab_desc S, unsigned long long *out)
{
    uint32_t freeobj = 0, freeslabs = 0;
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < S.nslabs; s += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = 0;
        for (uint32_t w = 0; w < kSlabWords; w++) c += __popcll((long long)S.bits[s * kSlabWords + w]);
        freeobj += c;
        freeslabs += c == kSlabObjects;
    }
    unsigned am = __activemask();
    freeobj = __reduce_add_sync(am, freeobj);
    freeslabs = __reduce_add_sync(am, freeslabs);
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(am) - 1)) {
        if (freeobj) atomicAdd(out, (unsigned long long)freeobj);
        if (freeslabs) atomicAdd(out + 1, (unsigned long long)freeslabs);
    }
}

struct set_desc {
    slab_desc s[PG_SLAB_MAX_CLASSES];
    uint64_t bytes[PG_SLAB_MAX_CLASSES];
    uint32_t n;
};

// size -> class: the smallest class whose objects hold `size` bytes, or n
__device__ __forceinline__ uint32_t class_of(const set_desc &D, uint64_t size)
{
    uint32_t c = 0;
    while (c < D.n && D.bytes[c] < size) c++;
    return c;
}

// One malloc per request.  The lanes of a warp that ask the same class claim
// together (one snapshot and atomicAnd serve them all), so the block first
// orders its 256 requests by class in shared memory: a warp then holds one or
// two classes instead of most of them, and a claim serves up to 32 objects.
// Results go back to each request's own place.
#ifndef PG_SET_MALLOC_SORT
#define PG_SET_MALLOC_SORT 1
#endif
__global__ void __launch_bounds__(256) k_set_malloc(set_desc D, uint64_t n, const uint32_t *sizes, void **out,
                                                    unsigned long long *fails)
{
    const uint64_t base = (uint64_t)blockIdx.x * blockDim.x;
    const uint64_t i = base + threadIdx.x;
#if PG_SET_MALLOC_SORT
    // classes 0 .. D.n - 1, D.n = too large for every class, D.n + 1 = no request
    __shared__ uint32_t cnt[PG_SLAB_MAX_CLASSES + 2];
    __shared__ uint8_t cls[256];
    __shared__ uint8_t from[256];
    if (threadIdx.x < PG_SLAB_MAX_CLASSES + 2) cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t c0 = i < n ? class_of(D, sizes[i]) : D.n + 1;
    const uint32_t rank = atomicAdd(&cnt[c0], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t at = 0;
        for (uint32_t c = 0; c < D.n + 2; c++) {
            const uint32_t k = cnt[c];
            cnt[c] = at;
            at += k;
        }
    }
    __syncthreads();
    cls[cnt[c0] + rank] = (uint8_t)c0;
    from[cnt[c0] + rank] = (uint8_t)threadIdx.x;
    __syncthreads();
    const uint32_t c = cls[threadIdx.x];
    const uint64_t dst = base + from[threadIdx.x];
    const unsigned peers = __match_any_sync(0xffffffffu, c);  // the lanes asking the same class claim together
    if (c > D.n) return;  // no request here (the block's tail)
#else
    if (i >= n) return;
    const uint32_t c = class_of(D, sizes[i]);
    const uint64_t dst = i;
    const unsigned peers = __match_any_sync(__activemask(), c);  // the lanes asking the same class claim together
#endif
    void *p = nullptr;
    if (c < D.n) {
        const uint64_t off = slab_claim(D.s[c], peers);
        if (off != ~0ULL) p = D.s[c].pool + off * D.s[c].size;
    }
    out[dst] = p;
    if (!p && fails) atomicAdd(fails, 1ULL);
}

__global__ void __launch_bounds__(256) k_set_free(set_desc D, uint64_t n, void *const *ptrs, unsigned long long *bad)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned char *p = (const unsigned char *)ptrs[i];
        if (!p) continue;
        bool ok = false;
        for (uint32_t c = 0; c < D.n; c++) {
            const slab_desc &S = D.s[c];
            if (p >= S.pool && p < S.pool + S.nslabs * kSlabObjects * S.size) {
                ok = slab_release(S, p);
                break;
            }
        }
        if (!ok && bad) atomicAdd(bad, 1ULL);
    }
}

unsigned grid_for(uint64_t n)
{
    uint64_t b = (n + 255) / 256;
    return (unsigned)(b ? b : 1);
}

}  // namespace

extern "C" {

pg_status pg_slab_create(uint64_t num_allocs, uint64_t object_bytes, pg_slab **out)
{
    if (!out || num_allocs == 0 || object_bytes == 0) return PG_ERR_INVALID;
    *out = nullptr;
    pg_slab *a = (pg_slab *)calloc(1, sizeof(pg_slab));
    if (!a) return PG_ERR_NOMEM;
    const uint64_t nslabs = (num_allocs - 1) / kSlabObjects + 1;  // slab_one_size.cuh:94
    if (nslabs > 0xFFFFFFFEull || object_bytes > ~0ull / (nslabs * kSlabObjects) ||
        cudaGetDevice(&a->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&a->num_sms, cudaDevAttrMultiProcessorCount, a->device) != cudaSuccess) {
        cudaGetLastError();
        free(a);
        return PG_ERR_INVALID;
    }
    a->d.nslabs = nslabs;
    a->d.size = object_bytes;
    a->capacity = nslabs * kSlabObjects;
    a->pool_bytes = a->capacity * object_bytes;
    const uint64_t nsum = (nslabs + 63) / 64;
    cudaError_t e = cudaMalloc(&a->d.pool, a->pool_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.bits, nslabs * kSlabWords * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.mgr, nslabs * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.summary, nsum * 8);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.cursor, kSlabCursors * 4);
    if (e == cudaSuccess) e = cudaMalloc(&a->d.stats, 2 * 8);
    if (e != cudaSuccess) {
        cudaGetLastError();
        pg_slab_destroy(a);
        return cuda_status(e);
    }

    {
        pg_status st = pg_slab_reset(a, nullptr);
        if (st != PG_OK) {
            pg_slab_destroy(a);
            return st;
        }
        if (cudaDeviceSynchronize() != cudaSuccess) {
            pg_slab_destroy(a);
            return PG_ERR_CUDA;
        }
    }
    *out = a;
    return PG_OK;
}

pg_status pg_slab_destroy(pg_slab *a)
{
    if (!a) return PG_ERR_INVALID;
    cudaFree(a->d.pool);
    cudaFree(a->d.bits);
    cudaFree(a->d.mgr);
    cudaFree(a->d.summary);
    cudaFree(a->d.cursor);
    cudaFree(a->d.stats);
    free(a);
    return PG_OK;
}

pg_status pg_slab_reset(pg_slab *a, pg_stream_t stream)
{
    if (!a || !pg_on_device(a->device)) return PG_ERR_INVALID;
    const uint64_t words = a->d.nslabs * kSlabWords;
    uint64_t blocks = (words + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_slab_init<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a->d);
    return cuda_status(cudaGetLastError());
}

pg_status pg_slab_info(const pg_slab *a, pg_slab_info_t *out)
{
    if (!a || !out) return PG_ERR_INVALID;
    out->pool = a->d.pool;
    out->pool_bytes = a->pool_bytes;
    out->object_bytes = a->d.size;
    out->capacity = a->capacity;
    out->nslabs = a->d.nslabs;
    out->d_stats = reinterpret_cast<uint64_t *>(a->d.stats);
    return PG_OK;
}

pg_status pg_slab_bulk_malloc(pg_slab *a, uint64_t n, void **d_ptrs, uint64_t *d_fail_count, pg_stream_t stream)
{
    if (!a || (n && !d_ptrs) || !pg_on_device(a->device)) return PG_ERR_INVALID;
    if (n == 0) return PG_OK;
    k_slab_malloc<<<grid_for(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        a->d, n, d_ptrs, reinterpret_cast<unsigned long long *>(d_fail_count));
    return cuda_status(cudaGetLastError());
}

pg_status pg_slab_desc(const pg_slab *a, void *out_desc, uint64_t bytes)
{
    if (!a || !out_desc || bytes != sizeof(slab_desc)) return PG_ERR_INVALID;
    memcpy(out_desc, &a->d, sizeof(slab_desc));
    return PG_OK;
}

pg_status pg_slab_bulk_free(pg_slab *a, void *const *d_ptrs, uint64_t n, uint64_t *d_bad_count, pg_stream_t stream)
{
    if (!a || (n && !d_ptrs) || !pg_on_device(a->device)) return PG_ERR_INVALID;
    if (n == 0) return PG_OK;
    uint64_t blocks = grid_for(n);
    if (blocks > (uint64_t)a->num_sms * 32) blocks = (uint64_t)a->num_sms * 32;
    k_slab_free<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        a->d, n, d_ptrs, reinterpret_cast<unsigned long long *>(d_bad_count));
    return cuda_status(cudaGetLastError());
}

pg_status pg_slab_count_free(pg_slab *a, uint64_t *d_out, pg_stream_t stream)
{
    if (!a || !d_out || !pg_on_device(a->device)) return PG_ERR_INVALID;
    uint64_t blocks = (a->d.nslabs + 255) / 256;
    if (blocks > (uint64_t)a->num_sms * 8) blocks = (uint64_t)a->num_sms * 8;
    k_slab_count<<<(unsigned)(blocks ? blocks : 1), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        a->d, reinterpret_cast<unsigned long long *>(d_out));
    return cuda_status(cudaGetLastError());
}

pg_status pg_slab_report(pg_slab *a, uint64_t *free_slabs, uint64_t *max_slabs, uint64_t *free_objects,
                         uint64_t *double_frees)
{
    if (!a || !pg_on_device(a->device)) return PG_ERR_INVALID;
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, 16) != cudaSuccess) return PG_ERR_NOMEM;
    pg_status st = cuda_status(cudaMemset(d, 0, 16));
    if (st == PG_OK) st = pg_slab_count_free(a, reinterpret_cast<uint64_t *>(d), nullptr);
    unsigned long long h[2] = {0, 0}, s[2] = {0, 0};
    if (st == PG_OK) st = cuda_status(cudaMemcpy(h, d, 16, cudaMemcpyDeviceToHost));
    if (st == PG_OK) st = cuda_status(cudaMemcpy(s, a->d.stats, 16, cudaMemcpyDeviceToHost));
    cudaFree(d);
    if (free_slabs) *free_slabs = h[1];
    if (max_slabs) *max_slabs = a->d.nslabs;
    if (free_objects) *free_objects = h[0];
    if (double_frees) *double_frees = s[0];
    return st;
}

pg_status pg_slab_set_create(uint32_t nclasses, const uint64_t *class_bytes, const uint64_t *num_allocs,
                             pg_slab_set **out)
{
    if (!out || !class_bytes || !num_allocs || nclasses == 0 || nclasses > PG_SLAB_MAX_CLASSES) return PG_ERR_INVALID;
    for (uint32_t c = 1; c < nclasses; c++)
        if (class_bytes[c] <= class_bytes[c - 1]) return PG_ERR_INVALID;
    pg_slab_set *s = (pg_slab_set *)calloc(1, sizeof(pg_slab_set));
    if (!s) return PG_ERR_NOMEM;
    for (uint32_t c = 0; c < nclasses; c++) {
        pg_status st = pg_slab_create(num_allocs[c], class_bytes[c], &s->cls[c]);
        if (st != PG_OK) {
            pg_slab_set_destroy(s);
            return st;
        }
        s->class_bytes[c] = class_bytes[c];
        s->nclasses = c + 1;
    }
    *out = s;
    return PG_OK;
}

pg_status pg_slab_set_destroy(pg_slab_set *s)
{
    if (!s) return PG_ERR_INVALID;
    for (uint32_t c = 0; c < PG_SLAB_MAX_CLASSES; c++)
        if (s->cls[c]) pg_slab_destroy(s->cls[c]);
    free(s);
    return PG_OK;
}

pg_slab *pg_slab_set_class(pg_slab_set *s, uint32_t c)
{
    return (s && c < s->nclasses) ? s->cls[c] : nullptr;
}

static set_desc make_set(const pg_slab_set *s)
{
    set_desc D;
    memset(&D, 0, sizeof(D));
    D.n = s->nclasses;
    for (uint32_t c = 0; c < s->nclasses; c++) {
        D.s[c] = s->cls[c]->d;
        D.bytes[c] = s->class_bytes[c];
    }
    return D;
}

pg_status pg_slab_set_bulk_malloc(pg_slab_set *s, const uint32_t *d_sizes, uint64_t n, void **d_ptrs,
                                  uint64_t *d_fail_count, pg_stream_t stream)
{
    if (!s || (n && (!d_ptrs || !d_sizes)) || !pg_on_device(s->cls[0]->device)) return PG_ERR_INVALID;
    if (n == 0) return PG_OK;
    k_set_malloc<<<grid_for(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        make_set(s), n, d_sizes, d_ptrs, reinterpret_cast<unsigned long long *>(d_fail_count));
    return cuda_status(cudaGetLastError());
}

pg_status pg_slab_set_bulk_free(pg_slab_set *s, void *const *d_ptrs, uint64_t n, uint64_t *d_bad_count,
                                pg_stream_t stream)
{
    if (!s || (n && !d_ptrs) || !pg_on_device(s->cls[0]->device)) return PG_ERR_INVALID;
    if (n == 0) return PG_OK;
    uint64_t blocks = grid_for(n);
    if (blocks > (uint64_t)s->cls[0]->num_sms * 32) blocks = (uint64_t)s->cls[0]->num_sms * 32;
    k_set_free<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        make_set(s), n, d_ptrs, reinterpret_cast<unsigned long long *>(d_bad_count));
    return cuda_status(cudaGetLastError());
}

}  // extern "C"
