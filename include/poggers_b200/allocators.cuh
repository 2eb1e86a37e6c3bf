// allocators.cuh -- the reference's slab allocator template API, implemented
// on the poggers_b200 slab pool.  Device code written against
//     poggers::allocators::one_size_slab_allocator<extra_blocks>
// (include/poggers/allocators/slab_one_size.cuh:58-659) compiles against
// poggers_b200::allocators::one_size_slab_allocator with the same host calls
// (generate_on_device(num_allocs, object_bytes) returning a device pointer,
// free_on_device, report_fill, report_max) and the same device calls
// (malloc(), free(ptr), get_offset_from_ptr, get_largest_allocation_offset,
// free_count_misses) and fields (offset_size, extra_memory).  The pool is
// created through the C ABI (pg_slab_create), so its bulk entry points can
// serve the same pool.
//
// extra_blocks is the reference's count of spare slabs kept per SM; slabs
// here are pinned per SM by a cursor and refilled from a summary bitmap, so
// the parameter is accepted and has no effect.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <cuda_runtime.h>
#include "poggers_b200.h"
#include "poggers_b200/slab.cuh"

namespace poggers_b200 {
namespace allocators {

template <int extra_blocks>
struct one_size_slab_allocator {
    using my_type = one_size_slab_allocator<extra_blocks>;
    uint64_t offset_size;  // object bytes (slab_one_size.cuh:63)
    char *extra_memory;    // object 0 of the pool (:65)
    pg::slab_desc desc;
    pg_slab *handle;

    // slab_one_size.cuh:84-141: a pool of ceil(num_allocs / 4096) slabs of
    // 4096 objects of ext_size bytes; throws like the reference when the
    // pool cannot be allocated
    static __host__ my_type *generate_on_device(uint64_t num_allocs, uint64_t ext_size)
    {
        pg_slab *h = nullptr;
        pg_status st = pg_slab_create(num_allocs, ext_size, &h);
        if (st != PG_OK) throw std::runtime_error("main malloc buffer failed to be acquired.\n");
        my_type host;
        host.handle = h;
        if (pg_slab_desc(h, &host.desc, sizeof(host.desc)) != PG_OK) {
            pg_slab_destroy(h);
            throw std::runtime_error("slab descriptor unavailable");
        }
        host.offset_size = ext_size;
        host.extra_memory = reinterpret_cast<char *>(host.desc.pool);
        my_type *dev = nullptr;
        if (cudaMalloc(&dev, sizeof(my_type)) != cudaSuccess) {
            pg_slab_destroy(h);
            throw std::runtime_error("cudaMalloc of the allocator descriptor failed");
        }
        cudaMemcpy(dev, &host, sizeof(my_type), cudaMemcpyHostToDevice);
        return dev;
    }

    static __host__ void free_on_device(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        pg_slab_destroy(host.handle);
        cudaFree(dev);
    }

    static __host__ pg_slab *host_handle(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        return host.handle;
    }

    // one object, or nullptr when none could be claimed within the bounded
    // attempts (the reference's SLAB_ONE_SIZE_MAX_ATTEMPTS, :20); callable by
    // any subset of a warp's threads, which are then served together
    __device__ void *malloc() { return pg::slab_malloc(desc); }

    // free (:428-464); a double free or a pointer that is not an object of
    // this pool is counted and ignored
    __device__ void free(void *ext_allocation) { pg::slab_release(desc, ext_allocation); }

    // free_count_misses (:466-506): misses += 1 when the free was refused
    __device__ void free_count_misses(void *ext_allocation, uint64_t *misses)
    {
        if (!pg::slab_release(desc, ext_allocation)) atomicAdd(reinterpret_cast<unsigned long long *>(misses), 1ULL);
    }

    __device__ uint64_t get_offset_from_ptr(void *ext_ptr)
    {
        return ((uint64_t)ext_ptr - (uint64_t)extra_memory) / offset_size;
    }

    // one past the largest object offset (:178-182)
    __device__ uint64_t get_largest_allocation_offset() { return desc.nslabs * pg::kSlabObjects; }

    // report_fill / report_max (:628-656): free slabs and slabs of the pool
    // (called on the device pointer, like the reference's)
    __host__ uint64_t report_fill()
    {
        uint64_t fs = 0, ms = 0, fo = 0, df = 0;
        pg_slab_report(host_handle(this), &fs, &ms, &fo, &df);
        return fs;
    }
    __host__ uint64_t report_max()
    {
        uint64_t fs = 0, ms = 0, fo = 0, df = 0;
        pg_slab_report(host_handle(this), &fs, &ms, &fo, &df);
        return ms;
    }
};

}  // namespace allocators
}  // namespace poggers_b200
