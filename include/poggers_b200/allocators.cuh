// allocators.cuh -- the reference's slab allocator template API, implemented
// on the poggers_b200 pinned slab pool.  Device code written against
//     poggers::allocators::one_size_slab_allocator<extra_blocks>
// (include/poggers/allocators/slab_one_size.cuh:58-659) compiles against
// poggers_b200::allocators::one_size_slab_allocator with the same host calls
// (generate_on_device(num_allocs, object_bytes) returning a device pointer,
// free_on_device, report_fill, report_max) and the same device calls
// (malloc(), free(ptr), free_count_misses, get_offset_from_ptr,
// get_largest_allocation_offset) and fields (offset_size, extra_memory).
//
// The pool follows the reference's slab policy (pg_pslab_*, slab_pinned.cuh):
// every SM pins a primary slab and extra_blocks backups when the pool is
// created, a malloc claims whole 64-object words and keeps the rest in its
// SM's cache, an exhausted primary is replaced by a backup and the backup's
// place refilled from the pool.  So, as with the reference, a pool needs room
// for those pins: ceil(num_allocs / 4096) slabs should exceed
// (extra_blocks + 1) x the SM count, or SMs without a slab return NULL (the
// reference's own tests add 15M objects to num_allocs for this,
// tests/src/slab_one_size_tests.cu:226).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <cuda_runtime.h>
#include "poggers_b200.h"
#include "poggers_b200/slab_pinned.cuh"

namespace poggers_b200 {
namespace allocators {

template <int extra_blocks>
struct one_size_slab_allocator {
    using my_type = one_size_slab_allocator<extra_blocks>;
    uint64_t offset_size;  // object bytes (slab_one_size.cuh:63)
    char *extra_memory;    // object 0 of the pool (:65)
    pg::pslab_desc desc;
    pg_pslab *handle;

    // slab_one_size.cuh:84-141: a pool of ceil(num_allocs / 4096) slabs of
    // 4096 objects of ext_size bytes, extra_blocks + 1 of them pinned to each
    // SM; throws like the reference when the pool cannot be allocated
    static __host__ my_type *generate_on_device(uint64_t num_allocs, uint64_t ext_size)
    {
        pg_pslab *h = nullptr;
        pg_status st = pg_pslab_create(num_allocs, ext_size, (uint32_t)extra_blocks, &h);
        if (st != PG_OK) throw std::runtime_error("main malloc buffer failed to be acquired.\n");
        my_type host;
        host.handle = h;
        if (pg_pslab_desc(h, &host.desc, sizeof(host.desc)) != PG_OK) {
            pg_pslab_destroy(h);
            throw std::runtime_error("slab descriptor unavailable");
        }
        host.offset_size = ext_size;
        host.extra_memory = reinterpret_cast<char *>(host.desc.pool);
        my_type *dev = nullptr;
        if (cudaMalloc(&dev, sizeof(my_type)) != cudaSuccess) {
            pg_pslab_destroy(h);
            throw std::runtime_error("cudaMalloc of the allocator descriptor failed");
        }
        cudaMemcpy(dev, &host, sizeof(my_type), cudaMemcpyHostToDevice);
        return dev;
    }

    static __host__ void free_on_device(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        pg_pslab_destroy(host.handle);
        cudaFree(dev);
    }

    static __host__ pg_pslab *host_handle(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        return host.handle;
    }

    // one object, or nullptr after SLAB_ONE_SIZE_MAX_ATTEMPTS (25, :20)
    // rounds; callable by any subset of a warp's threads, which are then
    // served together
    __device__ void *malloc() { return pg::pslab_malloc(desc); }

    // free (:428-464); a double free or a pointer that is not an object of
    // this pool changes nothing
    __device__ void free(void *ext_allocation) { pg::pslab_release(desc, ext_allocation); }

    // free_count_misses (:466-506): misses[0] += 1 when the free emptied an
    // unpinned slab and returned it to the pool, misses[1] += 1 when it
    // emptied a slab still pinned to an SM
    __device__ void free_count_misses(void *ext_allocation, uint64_t *misses)
    {
        const int r = pg::pslab_release(desc, ext_allocation);
        if (r == pg::PSLAB_RETURNED) atomicAdd(reinterpret_cast<unsigned long long *>(misses), 1ULL);
        else if (r == pg::PSLAB_EMPTIED_PINNED) atomicAdd(reinterpret_cast<unsigned long long *>(misses + 1), 1ULL);
    }

    __device__ uint64_t get_offset_from_ptr(void *ext_ptr)
    {
        return ((uint64_t)ext_ptr - (uint64_t)extra_memory) / offset_size;
    }

    // one past the largest object offset (:178-182)
    __device__ uint64_t get_largest_allocation_offset() { return desc.nslabs * pg::kPinnedObjects; }

    // report_fill / report_max (:628-656): slabs in the pool and slabs in all
    // (called on the device pointer, like the reference's)
    __host__ uint64_t report_fill()
    {
        uint64_t pool = 0, ms = 0, sms = 0, df = 0;
        pg_pslab_report(host_handle(this), &pool, &ms, &sms, &df);
        return pool;
    }
    __host__ uint64_t report_max()
    {
        uint64_t pool = 0, ms = 0, sms = 0, df = 0;
        pg_pslab_report(host_handle(this), &pool, &ms, &sms, &df);
        return ms;
    }
    // SM ids holding pins (no counterpart in the reference, which pins one
    // storage per SM of the device)
    __host__ uint64_t report_pinned_sms()
    {
        uint64_t pool = 0, ms = 0, sms = 0, df = 0;
        pg_pslab_report(host_handle(this), &pool, &ms, &sms, &df);
        return sms;
    }
};

}  // namespace allocators
}  // namespace poggers_b200
