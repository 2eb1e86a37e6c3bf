// test_bucketed_api.cu -- device callers of the bucketed filter written
// against the reference's template API, compiled against
// poggers_b200/tables.cuh.
//
// The table types are the reference's delete-test instantiations
// (tests/src/delete_tests.cu:138-179, del_TCF and del_TCF_small) spelled with
// this library's namespace, and the kernels follow that test's drivers
// (delete_tests.cu:248-460): one tile per key, insert, remove the first half,
// query the second half, re-add the first half with insert_with_delete, then
// insert_if_not_exists over present keys.  The filters are sized by that
// test's own generate_size (delete_tests.cu:771-779, a variadic_size of the
// primary and a 1 % backing level), spelled as there through the compat
// header's poggers namespace.  Prints one JSON line of counters.
#include <cstdio>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include "poggers_b200/compat.cuh"

namespace pb = poggers_b200;
namespace pr = pb::representations;

template <class SmallKey, int Bits>
using packed_rep = pr::dynamic_bucket_container<
    pr::dynamic_container<pr::bit_grouped_container<Bits, Bits>::template representation, SmallKey>::template representation>;

using del_backing_table = pb::tables::bucketed_table<uint64_t, uint16_t, packed_rep<uint16_t, 16>::template representation,
                                                     4, 8, pb::insert_schemes::linear_insert_bucket_scheme, 4000,
                                                     pb::probing_schemes::linearProber, pb::hashers::murmurHasher>;
using del_TCF = pb::tables::bucketed_table<uint64_t, uint16_t, packed_rep<uint16_t, 16>::template representation, 4, 16,
                                           pb::insert_schemes::power_of_n_insert_shortcut_bucket_scheme, 2,
                                           pb::probing_schemes::XORPowerOfTwoHasher, pb::hashers::murmurHasher, true,
                                           del_backing_table>;
using del_backing_table_small =
    pb::tables::bucketed_table<uint64_t, uint8_t, packed_rep<uint8_t, 8>::template representation, 4, 8,
                               pb::insert_schemes::linear_insert_bucket_scheme, 400, pb::probing_schemes::linearProber,
                               pb::hashers::murmurHasher>;
using del_TCF_small = pb::tables::bucketed_table<uint64_t, uint8_t, packed_rep<uint8_t, 8>::template representation, 4, 16,
                                                 pb::insert_schemes::power_of_n_insert_shortcut_bucket_scheme, 2,
                                                 pb::probing_schemes::XORPowerOfTwoHasher, pb::hashers::murmurHasher,
                                                 true, del_backing_table_small>;

template <class Filter, class Val>
__global__ void speed_insert_kernel(Filter *filter, const uint64_t *keys, const Val *vals, uint64_t n,
                                    unsigned long long *misses)
{
    auto tile = filter->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    if (!filter->insert(tile, keys[tid], vals[tid]) && tile.thread_rank() == 0) atomicAdd(misses, 1ULL);
}

template <class Filter, class Val>
__global__ void speed_insert_with_delete_kernel(Filter *filter, const uint64_t *keys, const Val *vals, uint64_t n,
                                                unsigned long long *misses)
{
    auto tile = filter->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    if (!filter->insert_with_delete(tile, keys[tid], vals[tid]) && tile.thread_rank() == 0) atomicAdd(misses, 1ULL);
}

template <class Filter, class Val>
__global__ void speed_delete_kernel(Filter *filter, const uint64_t *keys, uint64_t n, unsigned long long *misses)
{
    auto tile = filter->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    if (!filter->remove(tile, keys[tid]) && tile.thread_rank() == 0) atomicAdd(misses, 1ULL);
}

template <class Filter, class Val>
__global__ void speed_query_kernel(Filter *filter, const uint64_t *keys, const Val *vals, uint64_t n,
                                   unsigned long long *misses, unsigned long long *wrong)
{
    auto tile = filter->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    Val val = 0;
    bool r = filter->query(tile, keys[tid], val);
    if (tile.thread_rank() == 0) {
        if (!r) atomicAdd(misses, 1ULL);
        else if (val != vals[tid]) atomicAdd(wrong, 1ULL);
    }
}

template <class Filter, class Val>
__global__ void if_not_exists_kernel(Filter *filter, const uint64_t *keys, const Val *vals, uint64_t n,
                                     unsigned long long *not_found, unsigned long long *failed)
{
    auto tile = filter->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    Val ext = 0;
    bool found = false;
    bool r = filter->insert_if_not_exists(tile, keys[tid], (Val)(vals[tid] + 1), ext, found);
    if (tile.thread_rank() == 0) {
        if (!r) atomicAdd(failed, 1ULL);
        else if (!found) atomicAdd(not_found, 1ULL);
    }
}

static uint64_t splitmix(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// counters: 0 insert fails, 1 delete misses, 2 query misses, 3 query wrong values,
// 4 re-add fails, 5 if_not_exists not found, 6 if_not_exists failed
__host__ poggers::sizing::variadic_size generate_size(int nbits)
{
    uint64_t nslots = (1ULL << nbits);

    poggers::sizing::variadic_size internal_size(nslots, nslots / 100);

    return internal_size;
}

template <class Filter, class Val>
static int run(const char *name, int nbits, unsigned long long *bad, bool last)
{
    const uint64_t nslots = 1ULL << nbits;
    poggers::sizing::variadic_size size = generate_size(nbits);
    Filter *f = Filter::generate_on_device(&size, 42);
    const uint64_t num_slots = f->get_num_slots(), local_slots = f->get_local_num_slots();
    const uint64_t n = (uint64_t)(0.9 * (nslots + nslots / 100)), half = n / 2;
    std::vector<uint64_t> hk(n);
    std::vector<Val> hv(n);
    for (uint64_t i = 0; i < n; i++) {
        hk[i] = splitmix(42, i) | 1;  // never 0 (empty) in the 64-bit key
        hv[i] = (Val)splitmix(49, i);
    }
    uint64_t *dk;
    Val *dv;
    cudaMalloc(&dk, n * 8);
    cudaMalloc(&dv, n * sizeof(Val));
    cudaMemcpy(dk, hk.data(), n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, hv.data(), n * sizeof(Val), cudaMemcpyHostToDevice);
    cudaMemset(bad, 0, 8 * sizeof(unsigned long long));
    speed_insert_kernel<Filter, Val><<<Filter::get_num_blocks(n), Filter::get_block_size(n)>>>(f, dk, dv, n, bad + 0);
    const uint64_t fill_before = f->get_fill();
    speed_delete_kernel<Filter, Val><<<Filter::get_num_blocks(half), Filter::get_block_size(half)>>>(f, dk, half,
                                                                                                   bad + 1);
    const uint64_t fill_after = f->get_fill();
    speed_query_kernel<Filter, Val><<<Filter::get_num_blocks(n - half), Filter::get_block_size(n - half)>>>(
        f, dk + half, dv + half, n - half, bad + 2, bad + 3);
    speed_insert_with_delete_kernel<Filter, Val><<<Filter::get_num_blocks(half), Filter::get_block_size(half)>>>(
        f, dk, dv, half, bad + 4);
    const uint64_t fill_final = f->get_fill();
    if_not_exists_kernel<Filter, Val><<<Filter::get_num_blocks(n), Filter::get_block_size(n)>>>(f, dk, dv, n, bad + 5,
                                                                                              bad + 6);
    cudaError_t e = cudaDeviceSynchronize();
    unsigned long long h[8];
    cudaMemcpy(h, bad, sizeof(h), cudaMemcpyDeviceToHost);
    Filter::free_on_device(f);
    cudaFree(dk);
    cudaFree(dv);
    printf("\"%s\": {\"keys\": %llu, \"insert_fail\": %llu, \"delete_miss\": %llu, \"query_miss\": %llu, "
           "\"query_wrong_val\": %llu, \"readd_fail\": %llu, \"ine_not_found\": %llu, \"ine_fail\": %llu, "
           "\"fill_before\": %llu, \"fill_after_delete\": %llu, \"fill_final\": %llu, \"num_slots\": %llu, "
           "\"local_num_slots\": %llu, \"cuda\": %d}%s\n",
           name, (unsigned long long)n, h[0], h[1], h[2], h[3], h[4], h[5], h[6], (unsigned long long)fill_before,
           (unsigned long long)fill_after, (unsigned long long)fill_final, (unsigned long long)num_slots,
           (unsigned long long)local_slots, (int)e, last ? "" : ",");
    return e == cudaSuccess ? 0 : 1;
}

int main()
{
    unsigned long long *bad;
    cudaMalloc(&bad, 8 * sizeof(unsigned long long));
    printf("{\n");
    int rc = run<del_TCF, uint16_t>("del_TCF", 20, bad, false);
    rc |= run<del_TCF_small, uint8_t>("del_TCF_small", 20, bad, true);
    printf("}\n");
    cudaFree(bad);
    return rc;
}
