// ref_cuda_harness.cu -- TEST / BASELINE INFRASTRUCTURE: drives the REFERENCE's
// own CUDA tables (its headers, unmodified) with a C ABI, so the tests can
// take golden vectors from the reference and bench.py can time the reference
// CUDA build on the same GPU.
//
// Built by `make -C oracle refcuda` from the reference checkout (include path
// only) for sm_100a with -O3 and without the -G -g that the reference's CMake
// adds (CMakeLists.txt:50); the library lands in oracle/_ref/.
//
// Kernels follow the reference test drivers: one cooperative tile per key,
// 1024-thread blocks, Table::get_num_blocks (tests/src/test_mhm_tcf.cu:319-345,
// 457-521; tests/src/delete_tests.cu:336-372), with per-key result arrays in
// place of the drivers' global miss counters.  The serial shape (one tile, keys
// in order) mirrors tcf_find_first_fill / speed_insert_kernel_one_thread
// (test_mhm_tcf.cu:266-314, delete_tests.cu:298-333).
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include <poggers/data_structs/tcf.cuh>
#include <poggers/data_structs/uint64_hash_table.cuh>
#include <poggers/probing_schemes/power_of_two.cuh>
#include <poggers/probing_schemes/linear_probing.cuh>
#include <poggers/probing_schemes/xor_power_of_two.cuh>
#include <poggers/representations/dynamic_container.cuh>
#include <poggers/representations/grouped_storage_sub_bits.cuh>
#include <poggers/representations/packed_bucket.cuh>
#include <poggers/insert_schemes/power_of_n_shortcut_buckets.cuh>
#include <poggers/insert_schemes/linear_insert_buckets.cuh>
#include <poggers/sizing/default_sizing.cuh>
#include <poggers/tables/bucketed_table.cuh>

namespace pt = poggers::tables;
namespace pr = poggers::representations;
namespace pi = poggers::insert_schemes;
namespace pp = poggers::probing_schemes;
namespace ph = poggers::hashers;

// 0: the modular hash table of the bench workload: bucket 8, 20 double-hash probes
using ht_double_b8 = pt::static_table<uint64_t, uint64_t, pr::key_val_pair, 4, 8, pi::bucket_insert, 20,
                                      pp::doubleHasher, ph::murmurHasher>;
// 1: data_structs::hash_table_64 (bucket 16)
using ht_alias = poggers::data_structs::hash_table_64;
// 2: linear probing, bucket 8
using ht_linear_b8 = pt::static_table<uint64_t, uint64_t, pr::key_val_pair, 4, 8, pi::bucket_insert, 20,
                                      pp::linearProber, ph::murmurHasher>;
// 3: two-choice shortcut with power-of-two probing, bucket 8
using ht_p2_b8 = pt::static_table<uint64_t, uint64_t, pr::key_val_pair, 4, 8, pi::power_of_n_insert_shortcut_scheme,
                                  2, pp::powerOfTwoHasher, ph::murmurHasher>;
// 4: data_structs::tcf (two-choice, 16-slot buckets, backed by tiny_static_table_4)
using tcf_alias = poggers::data_structs::tcf;
// 5: tag-only two-choice filter (tests/src/bucket_speed_tests.cu tcqf_16_16)
using tcqf = pt::static_table<uint64_t, uint16_t, pr::dynamic_container<pr::key_container, uint16_t>::representation,
                              4, 16, pi::power_of_n_insert_shortcut_scheme, 2, pp::doubleHasher, ph::murmurHasher>;

// 6 / 7: the bucketed filters with tombstone reuse of tests/src/delete_tests.cu:138-179
// (del_TCF: 16-bit tags and values; del_TCF_small: 8-bit), primary two-choice
// shortcut over 16-slot packed buckets, backed by a linear-probing 8-slot table
template <class SmallKey, class Val, int Bits>
using packed_rep = pr::dynamic_bucket_container<
    pr::dynamic_container<pr::bit_grouped_container<Bits, Bits>::template representation, SmallKey>::template representation>;
using del_backing = pt::bucketed_table<uint64_t, uint16_t, packed_rep<uint16_t, uint16_t, 16>::template representation, 4, 8,
                                       pi::linear_insert_bucket_scheme, 4000, pp::linearProber, ph::murmurHasher>;
using del_tcf = pt::bucketed_table<uint64_t, uint16_t, packed_rep<uint16_t, uint16_t, 16>::template representation, 4, 16,
                                   pi::power_of_n_insert_shortcut_bucket_scheme, 2, pp::XORPowerOfTwoHasher,
                                   ph::murmurHasher, true, del_backing>;
using del_backing_small = pt::bucketed_table<uint64_t, uint8_t, packed_rep<uint8_t, uint8_t, 8>::template representation, 4,
                                             8, pi::linear_insert_bucket_scheme, 400, pp::linearProber,
                                             ph::murmurHasher>;
using del_tcf_small = pt::bucketed_table<uint64_t, uint8_t, packed_rep<uint8_t, uint8_t, 8>::template representation, 4, 16,
                                         pi::power_of_n_insert_shortcut_bucket_scheme, 2, pp::XORPowerOfTwoHasher,
                                         ph::murmurHasher, true, del_backing_small>;

// bucketed ops: 0 insert, 1 query, 2 remove, 3 insert_with_delete,
// 4 insert_if_not_exists, 5 insert_if_not_exists_delete
template <class T, class Val>
__device__ bool bop(T *table, cg::thread_block_tile<4> tile, int op, uint64_t key, Val val, Val &out, bool &found)
{
    switch (op) {
    case 0: return table->insert(tile, key, val);
    case 1: return table->query(tile, key, out);
    case 2: return table->remove(tile, key);
    case 3: return table->insert_with_delete(tile, key, val);
    case 4: return table->insert_if_not_exists(tile, key, val, out, found);
    default: return table->insert_if_not_exists_delete(tile, key, val, out, found);
    }
}

template <class T, class Val>
__global__ void ref_bop(T *table, int op, const uint64_t *keys, const Val *vals, uint64_t n, uint8_t *ok,
                        Val *vals_out, uint8_t *found, int serial)
{
    auto tile = table->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    uint64_t lo = tid, hi = tid + 1;
    if (serial) {
        if (tid != 0) return;
        lo = 0;
        hi = n;
    }
    for (uint64_t i = lo; i < hi && i < n; i++) {
        Val v = 0;
        bool f = false;
        bool r = bop<T, Val>(table, tile, op, keys[i], vals ? vals[i] : (Val)0, v, f);
        if (tile.thread_rank() == 0) {
            if (ok) ok[i] = r;
            if (vals_out) vals_out[i] = r ? v : (Val)0;
            if (found) found[i] = f;
        }
    }
}

template <class T, class Val>
static int bbulk_t(void *tp, int op, const uint64_t *keys, const void *vals, uint64_t n, uint8_t *ok, void *vals_out,
                   uint8_t *found, int serial, cudaStream_t s)
{
    T *t = static_cast<T *>(tp);
    if (n == 0) return 0;
    if (serial) {
        ref_bop<T, Val><<<1, 32, 0, s>>>(t, op, keys, (const Val *)vals, n, ok, (Val *)vals_out, found, 1);
    } else {
        uint64_t blocks = t->get_num_blocks(n), bs = t->get_block_size(n);
        ref_bop<T, Val><<<blocks, bs, 0, s>>>(t, op, keys, (const Val *)vals, n, ok, (Val *)vals_out, found, 0);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <class T>
static void *bcreate_t(uint64_t n0, uint64_t n1, uint64_t seed)
{
    poggers::sizing::size_in_num_slots<2> sz(n0, n1);
    return T::generate_on_device(&sz, seed);
}

template <class T, class Val>
__global__ void ref_insert(T *table, const uint64_t *keys, const Val *vals, uint64_t n, uint8_t *ok)
{
    auto tile = table->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    bool r = table->insert(tile, keys[tid], vals ? vals[tid] : (Val)0);
    if (tile.thread_rank() == 0 && ok) ok[tid] = r;
}

template <class T, class Val>
__global__ void ref_query(T *table, const uint64_t *keys, uint64_t n, Val *vals, uint8_t *found)
{
    auto tile = table->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    Val v = 0;
    bool r = table->query(tile, keys[tid], v);
    if (tile.thread_rank() == 0) {
        if (found) found[tid] = r;
        if (vals) vals[tid] = r ? v : (Val)0;
    }
}

template <class T>
__global__ void ref_remove(T *table, const uint64_t *keys, uint64_t n, uint8_t *ok)
{
    auto tile = table->get_my_tile();
    uint64_t tid = tile.meta_group_size() * blockIdx.x + tile.meta_group_rank();
    if (tid >= n) return;
    bool r = table->remove(tile, keys[tid]);
    if (tile.thread_rank() == 0 && ok) ok[tid] = r;
}

// one tile, keys in batch order
template <class T, class Val>
__global__ void ref_serial(T *table, int op, const uint64_t *keys, const Val *vals, uint64_t n, uint8_t *flags,
                           Val *vals_out)
{
    auto tile = table->get_my_tile();
    if (blockIdx.x != 0 || tile.meta_group_rank() != 0) return;
    for (uint64_t i = 0; i < n; i++) {
        bool r;
        Val v = 0;
        if (op == 0) r = table->insert(tile, keys[i], vals ? vals[i] : (Val)0);
        else if (op == 1) r = table->query(tile, keys[i], v);
        else r = table->remove(tile, keys[i]);
        if (tile.thread_rank() == 0) {
            if (flags) flags[i] = r;
            if (op == 1 && vals_out) vals_out[i] = r ? v : (Val)0;
        }
    }
}

// device struct layouts (all packed): static_table {scheme*, secondary*}
// (tables/base_table.cuh:70-72); bucket_insert and power_of_n_insert_shortcut_scheme
// {slots*, num_buckets, seed} (bucket_insert.cuh:46-49, power_of_n_shortcut.cuh:47-50)
struct raw_table { void *scheme; void *secondary; };
struct raw_scheme { void *slots; uint64_t num_buckets; uint64_t seed; };

struct handle {
    int kind;
    void *table;
};

template <class T>
static void *create_t(uint64_t n0, uint64_t n1, uint64_t seed, int levels)
{
    static_assert(sizeof(T) == sizeof(raw_table), "static_table layout");
    if (levels == 2) {
        poggers::sizing::size_in_num_slots<2> s(n0, n1);
        return T::generate_on_device(&s, seed);
    }
    poggers::sizing::size_in_num_slots<1> s(n0);
    return T::generate_on_device(&s, seed);
}

template <class T, class Val>
static int bulk_t(void *tp, int op, const uint64_t *keys, const void *vals, uint64_t n, uint8_t *flags, void *vals_out,
                  int serial, cudaStream_t s)
{
    T *t = static_cast<T *>(tp);
    if (n == 0) return 0;
    if (serial) {
        ref_serial<T, Val><<<1, 32, 0, s>>>(t, op, keys, (const Val *)vals, n, flags, (Val *)vals_out);
    } else {
        uint64_t blocks = T::get_num_blocks(n), bs = T::get_block_size(n);
        if (op == 0) ref_insert<T, Val><<<blocks, bs, 0, s>>>(t, keys, (const Val *)vals, n, flags);
        else if (op == 1) ref_query<T, Val><<<blocks, bs, 0, s>>>(t, keys, n, (Val *)vals_out, flags);
        else ref_remove<T><<<blocks, bs, 0, s>>>(t, keys, n, flags);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" {

// kind: see the aliases above; levels: 1 or 2 (kinds 4, 6 and 7 have a backing table)
void *refc_create(int kind, uint64_t n0, uint64_t n1, uint64_t seed)
{
    handle *h = new handle{kind, nullptr};
    switch (kind) {
    case 0: h->table = create_t<ht_double_b8>(n0, n1, seed, 1); break;
    case 1: h->table = create_t<ht_alias>(n0, n1, seed, 1); break;
    case 2: h->table = create_t<ht_linear_b8>(n0, n1, seed, 1); break;
    case 3: h->table = create_t<ht_p2_b8>(n0, n1, seed, 1); break;
    case 4: h->table = create_t<tcf_alias>(n0, n1, seed, 2); break;
    case 5: h->table = create_t<tcqf>(n0, n1, seed, 1); break;
    case 6: h->table = bcreate_t<del_tcf>(n0, n1, seed); break;
    case 7: h->table = bcreate_t<del_tcf_small>(n0, n1, seed); break;
    default: delete h; return nullptr;
    }
    cudaDeviceSynchronize();
    return h;
}

void refc_destroy(void *hp)
{
    handle *h = static_cast<handle *>(hp);
    switch (h->kind) {
    case 0: ht_double_b8::free_on_device((ht_double_b8 *)h->table); break;
    case 1: ht_alias::free_on_device((ht_alias *)h->table); break;
    case 2: ht_linear_b8::free_on_device((ht_linear_b8 *)h->table); break;
    case 3: ht_p2_b8::free_on_device((ht_p2_b8 *)h->table); break;
    case 4: tcf_alias::free_on_device((tcf_alias *)h->table); break;
    case 5: tcqf::free_on_device((tcqf *)h->table); break;
    case 6: del_tcf::free_on_device((del_tcf *)h->table); break;
    case 7: del_tcf_small::free_on_device((del_tcf_small *)h->table); break;
    }
    delete h;
}

// op: 0 insert, 1 query, 2 remove.  vals typed per table (uint64 HT, uint16 filters).
int refc_bulk(void *hp, int op, const uint64_t *keys, const void *vals, uint64_t n, uint8_t *flags, void *vals_out,
              int serial, void *stream)
{
    handle *h = static_cast<handle *>(hp);
    cudaStream_t s = (cudaStream_t)stream;
    switch (h->kind) {
    case 0: return bulk_t<ht_double_b8, uint64_t>(h->table, op, keys, vals, n, flags, vals_out, serial, s);
    case 1: return bulk_t<ht_alias, uint64_t>(h->table, op, keys, vals, n, flags, vals_out, serial, s);
    case 2: return bulk_t<ht_linear_b8, uint64_t>(h->table, op, keys, vals, n, flags, vals_out, serial, s);
    case 3: return bulk_t<ht_p2_b8, uint64_t>(h->table, op, keys, vals, n, flags, vals_out, serial, s);
    case 4: return bulk_t<tcf_alias, uint16_t>(h->table, op, keys, vals, n, flags, vals_out, serial, s);
    case 5: return bulk_t<tcqf, uint16_t>(h->table, op, keys, vals, n, flags, vals_out, serial, s);
    case 6: return bbulk_t<del_tcf, uint16_t>(h->table, op, keys, vals, n, flags, vals_out, nullptr, serial, s);
    case 7: return bbulk_t<del_tcf_small, uint8_t>(h->table, op, keys, vals, n, flags, vals_out, nullptr, serial, s);
    }
    return -1;
}

// Bucketed filters (kinds 6, 7): all six operations, with the found_val output.
int refc_bbulk(void *hp, int op, const uint64_t *keys, const void *vals, uint64_t n, uint8_t *ok, void *vals_out,
               uint8_t *found, int serial, void *stream)
{
    handle *h = static_cast<handle *>(hp);
    cudaStream_t s = (cudaStream_t)stream;
    if (op < 0 || op > 5) return -1;
    switch (h->kind) {
    case 6: return bbulk_t<del_tcf, uint16_t>(h->table, op, keys, vals, n, ok, vals_out, found, serial, s);
    case 7: return bbulk_t<del_tcf_small, uint8_t>(h->table, op, keys, vals, n, ok, vals_out, found, serial, s);
    }
    return -1;
}

// Level `level` (0 primary, 1 backing): slot array pointer and bucket count.
int refc_level(void *hp, int level, void **d_slots, uint64_t *nbuckets)
{
    handle *h = static_cast<handle *>(hp);
    raw_table t;
    if (cudaMemcpy(&t, h->table, sizeof(t), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (level == 1) {
        if (h->kind != 4 && h->kind != 6 && h->kind != 7) return -1;
        if (cudaMemcpy(&t, t.secondary, sizeof(t), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    }
    raw_scheme sc;
    if (cudaMemcpy(&sc, t.scheme, sizeof(sc), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    *d_slots = sc.slots;
    *nbuckets = sc.num_buckets;
    return 0;
}

int refc_dump(void *hp, int level, void *host_dst, uint64_t bytes)
{
    void *slots;
    uint64_t nb;
    if (refc_level(hp, level, &slots, &nb) != 0) return -1;
    return cudaMemcpy(host_dst, slots, bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

}  // extern "C"
