// test_device_api.cu -- device callers written against the reference's
// template API, compiled against poggers_b200/tables.cuh.
//
// Mirrors the reference's own drivers: test_components.cu:345-366
// (keys id*39, vals key*44, insert then query on the same tile) and the
// speed kernels of test_mhm_tcf.cu:319-345 / 457-521 (one tile per key,
// get_num_blocks / get_block_size launch shape).  Prints one JSON line of
// counters; every counter must be 0 except the ones named *_ok.
#include <cstdio>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include "poggers_b200/tables.cuh"

namespace pb = poggers_b200;

// test_components.cu:47 table_type (tile 8, bucket 8, 20 double-hash probes)
using table_type = pb::tables::static_table<uint64_t, uint64_t, pb::representations::key_val_pair, 8, 8,
                                            pb::insert_schemes::bucket_insert, 20, pb::probing_schemes::doubleHasher,
                                            pb::hashers::murmurHasher>;

__global__ void test_table(table_type *dev_table, uint64_t max_id, unsigned long long *bad)
{
    auto insert_tile = dev_table->get_my_tile();
    uint64_t my_id = insert_tile.meta_group_size() * blockIdx.x + insert_tile.meta_group_rank();
    if (my_id > max_id) return;
    uint64_t key = my_id * 39;
    uint64_t val = key * 44;
    uint64_t found_val = 0;
    bool ins = dev_table->insert(insert_tile, key, val);
    bool q = dev_table->query(insert_tile, key, found_val);
    if (insert_tile.thread_rank() == 0) {
        if (!ins) atomicAdd(bad + 0, 1ULL);
        if (!q) atomicAdd(bad + 1, 1ULL);
        if (found_val != val) atomicAdd(bad + 2, 1ULL);
    }
}

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
__global__ void speed_query_kernel(Filter *filter, const uint64_t *keys, const Val *vals, uint64_t n,
                                   unsigned long long *query_misses, unsigned long long *query_wrong)
{
    auto tile = filter->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    Val val = 0;
    bool r = filter->query(tile, keys[tid], val);
    if (tile.thread_rank() == 0) {
        if (!r) atomicAdd(query_misses, 1ULL);
        else if (val != vals[tid]) atomicAdd(query_wrong, 1ULL);
    }
}

static uint64_t splitmix(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int main()
{
    unsigned long long *bad;
    cudaMalloc(&bad, 8 * sizeof(unsigned long long));
    cudaMemset(bad, 0, 8 * sizeof(unsigned long long));

    // 1. known-answer test of test_components.cu
    pb::sizing::size_in_num_slots<1> first_size(1ULL << 20);
    table_type *dev_table = table_type::generate_on_device(&first_size, 15);
    const uint64_t max_id = 100000;
    test_table<<<table_type::get_num_blocks(max_id + 1), table_type::get_block_size(max_id + 1)>>>(dev_table, max_id,
                                                                                                   bad);
    cudaDeviceSynchronize();
    uint64_t bytes = pb::tables::static_table<uint64_t, uint64_t, pb::representations::key_val_pair, 8, 8,
                                              pb::insert_schemes::bucket_insert, 20, pb::probing_schemes::doubleHasher,
                                              pb::hashers::murmurHasher>::host_handle(dev_table) ? 1 : 0;
    table_type::free_on_device(dev_table);

    // 2. the TCF alias through the device API, then its bulk entry point on the same table
    using tcf = pb::data_structs::tcf;
    const uint64_t nslots = 1ULL << 20, n = (uint64_t)(0.85 * nslots);
    pb::sizing::size_in_num_slots<2> tcf_size(nslots, nslots / 100);
    tcf *filter = tcf::generate_on_device(&tcf_size, 42);
    std::vector<uint64_t> hk(n);
    std::vector<uint16_t> hv(n);
    for (uint64_t i = 0; i < n; i++) {
        hk[i] = splitmix(42, i);
        hv[i] = (uint16_t)(splitmix(49, i) % 64);
    }
    uint64_t *dk;
    uint16_t *dv;
    cudaMalloc(&dk, n * 8);
    cudaMalloc(&dv, n * 2);
    cudaMemcpy(dk, hk.data(), n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, hv.data(), n * 2, cudaMemcpyHostToDevice);
    speed_insert_kernel<tcf, uint16_t><<<tcf::get_num_blocks(n), tcf::get_block_size(n)>>>(filter, dk, dv, n, bad + 3);
    speed_query_kernel<tcf, uint16_t><<<tcf::get_num_blocks(n), tcf::get_block_size(n)>>>(filter, dk, dv, n, bad + 4,
                                                                                           bad + 5);
    // the same table through the C ABI: every key present
    uint64_t *hits;
    cudaMalloc(&hits, 8);
    cudaMemset(hits, 0, 8);
    pg_status st = pg_bulk_query(tcf::host_handle(filter), dk, n, nullptr, nullptr, hits, nullptr);
    cudaError_t e = cudaDeviceSynchronize();
    unsigned long long h[8];
    uint64_t bulk_hits = 0;
    cudaMemcpy(h, bad, sizeof(h), cudaMemcpyDeviceToHost);
    cudaMemcpy(&bulk_hits, hits, 8, cudaMemcpyDeviceToHost);
    tcf::free_on_device(filter);
    printf("{\"kat_insert_fail\": %llu, \"kat_query_miss\": %llu, \"kat_wrong_val\": %llu, "
           "\"tcf_insert_fail\": %llu, \"tcf_false_negative\": %llu, \"tcf_wrong_val_ok\": %llu, "
           "\"bulk_missing\": %llu, \"status\": %d, \"cuda\": %d, \"handle_ok\": %llu}\n",
           h[0], h[1], h[2], h[3], h[4], h[5], (unsigned long long)(n - bulk_hits), (int)st, (int)e,
           (unsigned long long)bytes);
    return (h[0] || h[1] || h[2] || h[4] || st != PG_OK || e != cudaSuccess || bulk_hits != n) ? 1 : 0;
}
