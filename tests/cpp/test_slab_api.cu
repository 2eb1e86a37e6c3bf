// test_slab_api.cu -- device callers of the slab allocator written against
// the reference's template API, compiled against poggers_b200/allocators.cuh.
//
// Follows the reference's own drivers (tests/src/slab_one_size_tests.cu:
// allocate_into_array, the duplicate check of allocate_into_array_bits, and
// free_from_array), on a pool provisioned as that test provisions it: every
// thread mallocs one object and writes into it, a bitmap over object offsets
// catches any object handed out twice, every object is freed with
// free_count_misses (slabs returned to the pool / emptied while pinned), the
// objects are allocated a second time, and a second free of one object is
// refused.  A third pass calls malloc() from three
// divergent branches of one warp (each branch its own call site, after
// different amounts of work), the way arbitrary device code may call it.
// Prints one JSON line.
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "poggers_b200/allocators.cuh"

namespace pb = poggers_b200;
using allocator = pb::allocators::one_size_slab_allocator<15>;

__global__ void allocate_into_array_bits(allocator *a, uint64_t *ptrs, uint64_t *bitmap, uint64_t n,
                                         unsigned long long *c)
{
    uint64_t tid = threadIdx.x + (uint64_t)blockIdx.x * blockDim.x;
    if (tid >= n) return;
    void *p = a->malloc();
    ptrs[tid] = (uint64_t)p;
    if (!p) {
        atomicAdd(c + 0, 1ULL);  // misses
        return;
    }
    ((char *)p)[0] = 't';
    uint64_t off = a->get_offset_from_ptr(p);
    if (off >= a->get_largest_allocation_offset()) atomicAdd(c + 1, 1ULL);  // out of the pool
    unsigned long long old = atomicOr((unsigned long long *)&bitmap[off / 64], 1ULL << (off % 64));
    if (old & (1ULL << (off % 64))) atomicAdd(c + 2, 1ULL);  // handed out twice
}

// malloc() from divergent code: the lanes of a warp split three ways by a hash
// of their index, do different amounts of work, and allocate at three call sites
__global__ void allocate_divergent(allocator *a, uint64_t *ptrs, uint64_t *bitmap, uint64_t n,
                                   unsigned long long *c)
{
    uint64_t tid = threadIdx.x + (uint64_t)blockIdx.x * blockDim.x;
    if (tid >= n) return;
    uint32_t h = (uint32_t)(tid * 2654435761ULL >> 7);
    void *p;
    uint32_t x = h;
    if (h % 3 == 0) {
        p = a->malloc();
    } else if (h % 3 == 1) {
        for (int i = 0; i < (int)(h & 15); ++i) x = x * 1664525u + 1013904223u;
        p = a->malloc();
    } else {
        for (int i = 0; i < 40 + (int)(h & 31); ++i) x = x * 22695477u + 1u;
        p = a->malloc();
    }
    ptrs[tid] = (uint64_t)p;
    if (!p) {
        atomicAdd(c + 0, 1ULL);
        return;
    }
    ((uint32_t *)p)[0] = x;
    uint64_t off = a->get_offset_from_ptr(p);
    if (off >= a->get_largest_allocation_offset()) atomicAdd(c + 1, 1ULL);
    unsigned long long old = atomicOr((unsigned long long *)&bitmap[off / 64], 1ULL << (off % 64));
    if (old & (1ULL << (off % 64))) atomicAdd(c + 2, 1ULL);
}

__global__ void free_from_array(allocator *a, uint64_t *ptrs, uint64_t n)
{
    uint64_t tid = threadIdx.x + (uint64_t)blockIdx.x * blockDim.x;
    if (tid >= n) return;
    void *p = (void *)ptrs[tid];
    if (p) a->free(p);
}

// free everything, counting with free_count_misses: misses[0] slabs returned
// to the pool, misses[1] slabs emptied while pinned
__global__ void free_from_array_counted(allocator *a, uint64_t *ptrs, uint64_t n, uint64_t *misses)
{
    uint64_t tid = threadIdx.x + (uint64_t)blockIdx.x * blockDim.x;
    if (tid >= n) return;
    void *p = (void *)ptrs[tid];
    if (p) a->free_count_misses(p, misses);
}

// the second free of one object is refused and counted by neither counter
__global__ void double_free(allocator *a, uint64_t *ptrs, uint64_t *misses)
{
    if (threadIdx.x + blockIdx.x * blockDim.x != 0) return;
    void *p = (void *)ptrs[0];
    a->free_count_misses(p, misses);
    a->free_count_misses(p, misses);
}

int main()
{
    // provisioned as the reference's own test (slab_one_size_tests.cu:226):
    // 15M objects beyond the ones allocated, for the slabs pinned to SMs
    const uint64_t n = 1ULL << 20;
    const uint64_t total = 15000000ULL + n + 4096;
    allocator *a = allocator::generate_on_device(total, 16);
    const uint64_t slabs = a->report_max(), fill_initial = a->report_fill(), sms = a->report_pinned_sms();
    uint64_t *ptrs, *bitmap;
    unsigned long long *c;
    cudaMalloc(&ptrs, n * 8);
    cudaMalloc(&bitmap, (slabs * 4096) / 8);
    cudaMalloc(&c, 16 * 8);
    cudaMemset(c, 0, 16 * 8);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    cudaMemset(bitmap, 0, (slabs * 4096) / 8);
    allocate_into_array_bits<<<blocks, 256>>>(a, ptrs, bitmap, n, c);
    cudaDeviceSynchronize();
    const uint64_t fill_full = a->report_fill();
    free_from_array_counted<<<blocks, 256>>>(a, ptrs, n, (uint64_t *)(c + 11));
    cudaDeviceSynchronize();
    const uint64_t fill_empty = a->report_fill();
    cudaMemset(bitmap, 0, (slabs * 4096) / 8);
    allocate_into_array_bits<<<blocks, 256>>>(a, ptrs, bitmap, n, c + 3);
    cudaDeviceSynchronize();
    free_from_array<<<blocks, 256>>>(a, ptrs, n);
    cudaMemset(bitmap, 0, (slabs * 4096) / 8);
    allocate_divergent<<<blocks, 256>>>(a, ptrs, bitmap, n, c + 8);
    cudaDeviceSynchronize();
    double_free<<<1, 32>>>(a, ptrs, (uint64_t *)(c + 6));
    cudaError_t e = cudaDeviceSynchronize();
    uint64_t pool = 0, ms = 0, ids = 0, doubles = 0;
    pg_pslab_report(allocator::host_handle(a), &pool, &ms, &ids, &doubles);
    unsigned long long h[16];
    cudaMemcpy(h, c, sizeof(h), cudaMemcpyDeviceToHost);
    allocator::free_on_device(a);
    cudaFree(ptrs);
    cudaFree(bitmap);
    cudaFree(c);
    printf("{\"allocs\": %llu, \"slabs\": %llu, \"sm_ids\": %llu, \"fill_initial\": %llu, \"misses\": %llu, "
           "\"out_of_pool\": %llu, \"duplicates\": %llu, \"fill_full\": %llu, \"returned\": %llu, "
           "\"emptied_pinned\": %llu, \"fill_empty\": %llu, \"misses_2\": %llu, \"out_of_pool_2\": %llu, "
           "\"duplicates_2\": %llu, \"misses_divergent\": %llu, \"out_of_pool_divergent\": %llu, "
           "\"duplicates_divergent\": %llu, \"double_free_counted\": %llu, \"double_free_seen\": %llu, "
           "\"cuda\": %d}\n",
           (unsigned long long)n, (unsigned long long)slabs, (unsigned long long)sms, (unsigned long long)fill_initial,
           h[0], h[1], h[2], (unsigned long long)fill_full, h[11], h[12], (unsigned long long)fill_empty, h[3], h[4],
           h[5], h[8], h[9], h[10], h[6] + h[7], (unsigned long long)doubles, (int)e);
    const bool ok = e == cudaSuccess && !h[0] && !h[1] && !h[2] && !h[3] && !h[4] && !h[5] && !h[8] && !h[9] &&
                    !h[10] && h[6] + h[7] == 0 && doubles == 1;
    return ok ? 0 : 1;
}
