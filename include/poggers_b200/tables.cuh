// tables.cuh -- the reference's template table API, implemented on the
// poggers_b200 bucket kernels.  Device code written against
//     poggers::tables::static_table<Key, Val, Rep, Partition_Size, Bucket_Size,
//                                   Insert_Scheme, Max_Probes, Probing_Scheme,
//                                   Hasher, Is_Recursive, Recursive_Type>
// (include/poggers/tables/base_table.cuh:52-356) compiles against
// poggers_b200::tables::static_table with the same template arguments, the
// same host calls (generate_on_device(Sizing*, seed) returning a device
// pointer, free_on_device, get_block_size, get_num_blocks, host_bytes_in_use)
// and the same device calls on a cooperative-groups tile (insert, query,
// remove, get_my_tile).  Tables are created through the C ABI
// (pg_table_create), so a table made here can also be driven by the bulk
// entry points.
//
// tables::bucketed_table (tables/bucketed_table.cuh:63-558) likewise, for the
// bucketed filter with tombstone reuse (dynamic_bucket_container of
// grouped_bits_pair<16,16> or <8,8> slots, power_of_n_insert_shortcut_bucket_scheme
// / linear_insert_bucket_scheme), with insert_with_delete and
// insert_if_not_exists[_delete] besides insert / query / remove.
//
// Supported instantiations (what the hot path uses): Key = uint64_t;
//   Rep key_val_pair with Val = uint64_t                 -> uint64 hash tables
//   Rep dynamic_container<key_val_pair, uint16_t>        -> TCF (16-bit tag + val)
//   Rep dynamic_container<key_container, uint16_t>       -> tag-only TCF
// Insert_Scheme bucket_insert or power_of_n_insert_shortcut_scheme; Probing
// doubleHasher, linearProber, powerOfTwoHasher or XORPowerOfTwoHasher; Hasher
// murmurHasher; Bucket_Size 4/8/16/32 on the primary level; at most one
// recursive (backing) table.
#pragma once
#include <cooperative_groups.h>
#include <stdexcept>
#include <vector>
#include <cstdint>
#include <cstddef>
#include "poggers_b200.h"
#include "poggers_b200/level.cuh"
#include "poggers_b200/packed.cuh"

namespace poggers_b200 {

namespace hashers {
template <typename Key, std::size_t Partition_size = 1>
struct murmurHasher {};
}  // namespace hashers

namespace representations {
template <typename Key, typename Val>
struct key_val_pair {};
template <typename Key, typename Val>
struct key_container {};
template <template <typename, typename> class Container, typename SmallKey>
struct dynamic_container {
    template <typename Key, typename Val>
    struct representation {};
};
// the bucketed filter's slot and bucket (grouped_storage_sub_bits.cuh:101-255,
// packed_bucket.cuh:29-278): bit_grouped_container<K, V>::representation is a
// packed (tag, value) word, dynamic_bucket_container<C>::representation a
// bucket of them with the tile width and bucket size as parameters
template <std::size_t key_bits, std::size_t val_bits>
struct bit_grouped_container {
    template <typename Key, typename Val>
    struct representation {};
};
template <template <typename, typename> class Container>
struct dynamic_bucket_container {
    template <typename Key, typename Val, std::size_t Partition_Size, std::size_t Bucket_Size>
    struct representation {};
};
}  // namespace representations

namespace probing_schemes {
template <typename Key, std::size_t P, template <typename, std::size_t> class H, std::size_t M>
struct doubleHasher {};
template <typename Key, std::size_t P, template <typename, std::size_t> class H, std::size_t M>
struct linearProber {};
template <typename Key, std::size_t P, template <typename, std::size_t> class H, std::size_t M>
struct powerOfTwoHasher {};
template <typename Key, std::size_t P, template <typename, std::size_t> class H, std::size_t M>
struct XORPowerOfTwoHasher {};
}  // namespace probing_schemes

namespace insert_schemes {
#define PG_SCHEME_PARAMS                                                                                       \
    typename Key, typename Val, std::size_t P, std::size_t B, template <typename, typename> class Rep, std::size_t M, \
        template <typename, std::size_t> class H,                                                              \
        template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class Probe
template <PG_SCHEME_PARAMS>
struct bucket_insert {};
template <PG_SCHEME_PARAMS>
struct power_of_n_insert_shortcut_scheme {};
#undef PG_SCHEME_PARAMS
// schemes over buckets of packed slots (power_of_n_shortcut_buckets.cuh,
// linear_insert_buckets.cuh): the representation takes the tile width and
// bucket size as parameters
#define PG_BSCHEME_PARAMS                                                                                          \
    typename Key, typename Val, std::size_t P, std::size_t B,                                                      \
        template <typename, typename, std::size_t, std::size_t> class Rep, std::size_t M,                          \
        template <typename, std::size_t> class H,                                                                  \
        template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class Probe
template <PG_BSCHEME_PARAMS>
struct power_of_n_insert_shortcut_bucket_scheme {};
template <PG_BSCHEME_PARAMS>
struct linear_insert_bucket_scheme {};
}  // namespace insert_schemes

namespace sizing {
// size_in_num_slots<N>: one slot count per table level (default_sizing.cuh:30-95)
template <std::size_t Num_Tables>
struct size_in_num_slots {
    uint64_t slots[Num_Tables];
    uint64_t i = 0;
    template <class... T>
    explicit size_in_num_slots(T... s) : slots{(uint64_t)s...}
    {
        static_assert(sizeof...(T) == Num_Tables, "one slot count per level");
    }
    uint64_t next() { return ++i <= Num_Tables ? slots[i - 1] : end(); }
    void reset() { i = 0; }
    uint64_t end() const { return ~uint64_t(0); }
    uint64_t total() const
    {
        uint64_t t = 0;
        for (std::size_t j = 0; j < Num_Tables; j++) t += slots[j];
        return t;
    }
};

// variadic_size: one slot count per table level, as many as the constructor is
// given (variadic_sizing.cuh:40-108), e.g. variadic_size(nslots, nslots / 100)
// for a filter and its backing table.  The counts live in a vector, so the
// object can be returned and copied by value; the cursor starts at the first
// count.
struct variadic_size {
    std::vector<uint64_t> slots;
    uint64_t i = 0;
    template <class... T>
    variadic_size(T... s) : slots{(uint64_t)s...}
    {
    }
    uint64_t next() { return ++i <= slots.size() ? slots[i - 1] : end(); }
    void reset() { i = 0; }
    uint64_t end() const { return ~uint64_t(0); }
    uint64_t total() const
    {
        uint64_t t = 0;
        for (uint64_t s : slots) t += s;
        return t;
    }
};
}  // namespace sizing

namespace detail {
template <template <typename, typename> class Rep, typename Val>
struct format_of;
template <>
struct format_of<representations::key_val_pair, uint64_t> { static constexpr uint32_t value = PG_FMT_KV64; };
template <template <typename, typename> class C, typename S>
struct is_dyn {};

template <template <typename, typename> class Rep>
struct rep_kind { static constexpr int value = -1; };
template <>
struct rep_kind<representations::key_val_pair> { static constexpr int value = 0; };
template <>
struct rep_kind<representations::dynamic_container<representations::key_val_pair, uint16_t>::template representation> {
    static constexpr int value = 1;
};
template <>
struct rep_kind<representations::dynamic_container<representations::key_container, uint16_t>::template representation> {
    static constexpr int value = 2;
};

template <template <typename, typename, std::size_t, std::size_t, template <typename, typename> class, std::size_t,
                    template <typename, std::size_t> class,
                    template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class>
          class S>
struct scheme_id { static constexpr int value = -1; };
template <>
struct scheme_id<insert_schemes::bucket_insert> { static constexpr int value = PG_SCHEME_BUCKET; };
template <>
struct scheme_id<insert_schemes::power_of_n_insert_shortcut_scheme> { static constexpr int value = PG_SCHEME_TWO_CHOICE; };

template <template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class Pr>
struct probe_id { static constexpr int value = -1; };
template <>
struct probe_id<probing_schemes::doubleHasher> { static constexpr int value = PG_PROBE_DOUBLE; };
template <>
struct probe_id<probing_schemes::linearProber> { static constexpr int value = PG_PROBE_LINEAR; };
template <>
struct probe_id<probing_schemes::powerOfTwoHasher> { static constexpr int value = PG_PROBE_P2; };
template <>
struct probe_id<probing_schemes::XORPowerOfTwoHasher> { static constexpr int value = PG_PROBE_XOR_P2; };
// packed formats: dynamic_bucket_container<dynamic_container<bit_grouped_container<W, W>, uintW>>
template <template <typename, typename, std::size_t, std::size_t> class Rep>
struct packed_bits { static constexpr int value = -1; };
template <>
struct packed_bits<representations::dynamic_bucket_container<representations::dynamic_container<
    representations::bit_grouped_container<16, 16>::template representation, uint16_t>::template representation>::
                       template representation> { static constexpr int value = 16; };
template <>
struct packed_bits<representations::dynamic_bucket_container<representations::dynamic_container<
    representations::bit_grouped_container<8, 8>::template representation, uint8_t>::template representation>::
                       template representation> { static constexpr int value = 8; };

template <template <typename, typename, std::size_t, std::size_t, template <typename, typename, std::size_t, std::size_t> class,
                    std::size_t, template <typename, std::size_t> class,
                    template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class>
          class S>
struct bscheme_id { static constexpr int value = -1; };
template <>
struct bscheme_id<insert_schemes::power_of_n_insert_shortcut_bucket_scheme> {
    static constexpr int value = PG_SCHEME_TWO_CHOICE_BUCKETED;
};
template <>
struct bscheme_id<insert_schemes::linear_insert_bucket_scheme> { static constexpr int value = PG_SCHEME_LINEAR_BUCKETED; };
}  // namespace detail

namespace tables {

// terminal of the recursion, like recursive_end_table (tables/recursive_end_table.cuh)
struct recursive_end_table {
    static constexpr bool kIsTable = false;
};

template <typename Key, typename Val, template <typename, typename> class Internal_Rep, std::size_t Partition_Size,
          std::size_t Bucket_Size,
          template <typename, typename, std::size_t, std::size_t, template <typename, typename> class, std::size_t,
                    template <typename, std::size_t> class,
                    template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class>
          class Insert_Scheme,
          std::size_t Max_Probes,
          template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class Probing_Scheme,
          template <typename, std::size_t> class Hasher, bool Is_Recursive = false,
          typename Recursive_Type = recursive_end_table>
struct static_table {
    static constexpr bool kIsTable = true;
    using key_type = Key;
    using val_type = Val;
    using my_type = static_table;
    static constexpr int kFmt = detail::rep_kind<Internal_Rep>::value;
    static constexpr int kScheme = detail::scheme_id<Insert_Scheme>::value;
    static constexpr int kProbe = detail::probe_id<Probing_Scheme>::value;
    static constexpr int G = (int)Partition_Size;
    static constexpr int B = (int)Bucket_Size;
    static_assert(std::is_same<Key, uint64_t>::value, "keys are uint64_t");
    static_assert(kFmt >= 0, "representation not supported on this path");
    static_assert(kFmt != 0 || std::is_same<Val, uint64_t>::value, "key_val_pair tables map uint64_t -> uint64_t");
    static_assert(kFmt == 0 || std::is_same<Val, uint16_t>::value, "filters carry uint16_t values");
    static_assert(kScheme >= 0 && kProbe >= 0, "insert / probing scheme not supported on this path");
    static_assert(B == 4 || B == 8 || B == 16 || B == 32, "primary bucket size 4, 8, 16 or 32");
    static_assert(G == 1 || G == 2 || G == 4 || G == 8 || G == 16, "tile of 1..16 lanes");
    using ops = pg::table_ops<kFmt, B, G, kScheme, Is_Recursive>;
    using dev_val = typename pg::fmt_t<kFmt>::V;

    pg::table_desc desc;
    pg_table *handle;

    static void fill_level(pg_level_config &L, uint64_t nslots)
    {
        L.nslots = nslots;
        L.bucket_size = (uint32_t)Bucket_Size;
        L.max_probes = (uint32_t)Max_Probes;
        L.scheme = (uint32_t)kScheme;
        L.probe = (uint32_t)kProbe;
    }

    template <typename Sizing_Type>
    static pg_table_config config_from(Sizing_Type *sizing)
    {
        pg_table_config c{};
        c.format = (uint32_t)kFmt;
        c.tile = (uint32_t)Partition_Size;
        c.nlevels = Is_Recursive ? 2 : 1;
        uint64_t n0 = sizing->next();
        if (n0 == sizing->end())
            throw std::runtime_error("Hash Table expects a num_slots from the sizing, but the size container is empty\n");
        fill_level(c.levels[0], n0);
        if constexpr (Is_Recursive) {
            static_assert(Recursive_Type::kIsTable, "recursive table type");
            uint64_t n1 = sizing->next();
            if (n1 == sizing->end())
                throw std::runtime_error("Hash Table expects a num_slots from the sizing, but the size container is empty\n");
            Recursive_Type::fill_level(c.levels[1], n1);
            c.levels[1].scheme = (uint32_t)Recursive_Type::kScheme;
            c.levels[1].probe = (uint32_t)Recursive_Type::kProbe;
        }
        if (sizing->next() != sizing->end())
            throw std::runtime_error("Hash Table Does not expect recursion but the size container is not empty.\n");
        return c;
    }

    // static_table::generate_on_device (base_table.cuh:110-145): returns a device pointer
    template <typename Sizing_Type>
    __host__ static my_type *generate_on_device(Sizing_Type *sizing, uint64_t seed)
    {
        pg_table_config c = config_from(sizing);
        pg_table *h = nullptr;
        pg_status st = pg_table_create(&c, seed, &h);
        if (st != PG_OK) throw std::runtime_error(pg_status_string(st));
        my_type host;
        host.handle = h;
        pg_level_info info;
        // the descriptor the bulk kernels use, rebuilt here for device callers
        for (uint32_t l = 0; l < c.nlevels; l++) {
            pg_table_level_info(h, l, &info);
            pg::level_desc &D = host.desc.lv[l];
            const pg_level_config &L = c.levels[l];
            const uint32_t kb = kFmt == 0 ? 8u : 2u, vb = kFmt == 0 ? 8u : (kFmt == 1 ? 2u : 0u);
            D.base = (unsigned char *)info.d_buckets;
            D.nbmod = pg::make_fastmod64(info.nbuckets);
            D.seed = info.seed;
            D.seed2 = info.seed * info.seed;
            D.bucket_size = L.bucket_size;
            D.max_probes = L.max_probes;
            D.scheme = L.scheme;
            D.probe = L.probe;
            D.bucket_bytes = L.bucket_size * (kb + vb);
        }
        host.desc.nlevels = c.nlevels;
        host.desc.format = (uint32_t)kFmt;
        my_type *dev = nullptr;
        if (cudaMalloc(&dev, sizeof(my_type)) != cudaSuccess) {
            pg_table_destroy(h);
            throw std::runtime_error("cudaMalloc of the table descriptor failed");
        }
        cudaMemcpy(dev, &host, sizeof(my_type), cudaMemcpyHostToDevice);
        return dev;
    }

    __host__ static void free_on_device(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        pg_table_destroy(host.handle);
        cudaFree(dev);
    }

    // the C-ABI handle behind a device pointer (to call the bulk entry points)
    __host__ static pg_table *host_handle(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        return host.handle;
    }

    __device__ __forceinline__ pg::group<G> group_of(const cooperative_groups::thread_block_tile<Partition_Size> &) const
    {
        return pg::group<G>::make();
    }

    __device__ bool insert(cooperative_groups::thread_block_tile<Partition_Size> tile, Key key, Val val)
    {
        return ops::insert(desc, group_of(tile), key, (dev_val)val);
    }
    __device__ bool insert(cooperative_groups::thread_block_tile<Partition_Size> tile, Key key)
    {
        return insert(tile, key, Val(0));
    }
    __device__ bool query(cooperative_groups::thread_block_tile<Partition_Size> tile, Key key, Val &val)
    {
        dev_val v = 0;
        bool r = ops::query(desc, group_of(tile), key, v);
        if (r) val = (Val)v;
        return r;
    }
    __device__ bool remove(cooperative_groups::thread_block_tile<Partition_Size> tile, Key key)
    {
        return ops::remove(desc, group_of(tile), key);
    }

    __device__ __inline__ cooperative_groups::thread_block_tile<Partition_Size> get_my_tile()
    {
        return cooperative_groups::tiled_partition<Partition_Size>(cooperative_groups::this_thread_block());
    }
    __host__ static uint64_t get_block_size(uint64_t) { return 1024; }
    __host__ static uint64_t get_num_blocks(uint64_t n) { return (Partition_Size * n - 1) / get_block_size(n) + 1; }
    __host__ uint64_t host_bytes_in_use() { return pg_table_bytes(host_handle(this)); }
};

// bucketed_table (tables/bucketed_table.cuh:63-558): the filter with
// tombstone reuse over buckets of packed (tag, value) words, with
// insert_with_delete and insert_if_not_exists[_delete] besides insert /
// query / remove.  Same host calls as static_table, plus get_fill.
template <typename Key, typename Val, template <typename, typename, std::size_t, std::size_t> class Internal_Rep,
          std::size_t Partition_Size, std::size_t Bucket_Size,
          template <typename, typename, std::size_t, std::size_t,
                    template <typename, typename, std::size_t, std::size_t> class, std::size_t,
                    template <typename, std::size_t> class,
                    template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class>
          class Insert_Scheme,
          std::size_t Max_Probes,
          template <typename, std::size_t, template <typename, std::size_t> class, std::size_t> class Probing_Scheme,
          template <typename, std::size_t> class Hasher, bool Is_Recursive = false,
          typename Recursive_Type = recursive_end_table>
struct bucketed_table {
    static constexpr bool kIsTable = true;
    using key_type = Key;
    using val_type = Val;
    using my_type = bucketed_table;
    static constexpr int kBits = detail::packed_bits<Internal_Rep>::value;
    static constexpr int kScheme = detail::bscheme_id<Insert_Scheme>::value;
    static constexpr int kProbe = detail::probe_id<Probing_Scheme>::value;
    static constexpr int G = (int)Partition_Size;
    static constexpr int B = (int)Bucket_Size;
    static_assert(std::is_same<Key, uint64_t>::value, "keys are uint64_t");
    static_assert(kBits > 0, "representation: dynamic_bucket_container of grouped_bits_pair<16,16> or <8,8>");
    static_assert((kBits == 16 && std::is_same<Val, uint16_t>::value) || (kBits == 8 && std::is_same<Val, uint8_t>::value),
                  "values are as wide as the tags");
    static_assert(kScheme >= 0 && kProbe >= 0, "insert / probing scheme not supported on this path");
    static_assert(B == 8 || B == 16 || B == 32, "bucket size 8, 16 or 32");
    static_assert(G == 1 || G == 2 || G == 4 || G == 8, "tile of 1..8 lanes");
    static constexpr int backing_bucket()
    {
        if constexpr (Is_Recursive) return Recursive_Type::B;
        else return 8;
    }
    static constexpr int B1 = backing_bucket();
    static_assert(B1 == 8 || B1 == 16, "backing bucket size 8 or 16");
    using tbl = pg::packed_table<kBits, B, B1, G, Is_Recursive>;

    pg::table_desc desc;
    pg_table *handle;

    static void fill_level(pg_level_config &L, uint64_t nslots)
    {
        L.nslots = nslots;
        L.bucket_size = (uint32_t)Bucket_Size;
        L.max_probes = (uint32_t)Max_Probes;
        L.scheme = (uint32_t)kScheme;
        L.probe = (uint32_t)kProbe;
    }

    template <typename Sizing_Type>
    static pg_table_config config_from(Sizing_Type *sizing)
    {
        pg_table_config c{};
        c.format = kBits == 16 ? (uint32_t)PG_FMT_PACKED_TAGVAL16 : (uint32_t)PG_FMT_PACKED_TAGVAL8;
        c.tile = (uint32_t)Partition_Size;
        c.nlevels = Is_Recursive ? 2 : 1;
        uint64_t n0 = sizing->next();
        if (n0 == sizing->end())
            throw std::runtime_error("Hash Table expects a num_slots from the sizing, but the size container is empty\n");
        fill_level(c.levels[0], n0);
        if constexpr (Is_Recursive) {
            static_assert(Recursive_Type::kIsTable && Recursive_Type::kBits == kBits, "recursive table of the same slots");
            uint64_t n1 = sizing->next();
            if (n1 == sizing->end())
                throw std::runtime_error("Hash Table expects a num_slots from the sizing, but the size container is empty\n");
            Recursive_Type::fill_level(c.levels[1], n1);
        }
        if (sizing->next() != sizing->end())
            throw std::runtime_error("Hash Table Does not expect recursion but the size container is not empty.\n");
        return c;
    }

    // bucketed_table::generate_on_device (bucketed_table.cuh:120-160): returns a device pointer
    template <typename Sizing_Type>
    __host__ static my_type *generate_on_device(Sizing_Type *sizing, uint64_t seed)
    {
        pg_table_config c = config_from(sizing);
        pg_table *h = nullptr;
        pg_status st = pg_table_create(&c, seed, &h);
        if (st != PG_OK) throw std::runtime_error(pg_status_string(st));
        my_type host;
        host.handle = h;
        pg_level_info info;
        for (uint32_t l = 0; l < c.nlevels; l++) {
            pg_table_level_info(h, l, &info);
            pg::level_desc &D = host.desc.lv[l];
            const pg_level_config &L = c.levels[l];
            D.base = (unsigned char *)info.d_buckets;
            D.nbmod = pg::make_fastmod64(info.nbuckets);
            D.seed = info.seed;
            D.seed2 = info.seed * info.seed;
            D.bucket_size = L.bucket_size;
            D.max_probes = L.max_probes;
            D.scheme = L.scheme;
            D.probe = L.probe;
            D.bucket_bytes = L.bucket_size * (uint32_t)(kBits / 4);
            D.fp = nullptr;
        }
        host.desc.nlevels = c.nlevels;
        host.desc.format = kBits == 16 ? (uint32_t)pg::FMT_PACKED16 : (uint32_t)pg::FMT_PACKED8;
        my_type *dev = nullptr;
        if (cudaMalloc(&dev, sizeof(my_type)) != cudaSuccess) {
            pg_table_destroy(h);
            throw std::runtime_error("cudaMalloc of the table descriptor failed");
        }
        cudaMemcpy(dev, &host, sizeof(my_type), cudaMemcpyHostToDevice);
        return dev;
    }

    __host__ static void free_on_device(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        pg_table_destroy(host.handle);
        cudaFree(dev);
    }

    __host__ static pg_table *host_handle(my_type *dev)
    {
        my_type host;
        cudaMemcpy(&host, dev, sizeof(my_type), cudaMemcpyDeviceToHost);
        return host.handle;
    }

    __device__ __forceinline__ bool run(int op, Key key, Val val, Val &out, bool &found) const
    {
        typename pg::pk<kBits>::V o = 0;
        const bool r = tbl::op(desc, pg::group<G>::make(), op, key, (uint64_t)val, o, found);
        out = (Val)o;
        return r;
    }

    __device__ bool insert(cooperative_groups::thread_block_tile<Partition_Size>, Key key, Val val)
    {
        Val o;
        bool f;
        return run(pg::POP_INSERT, key, val, o, f);
    }
    __device__ bool insert(cooperative_groups::thread_block_tile<Partition_Size> tile, Key key)
    {
        return insert(tile, key, Val(0));
    }
    __device__ bool insert_with_delete(cooperative_groups::thread_block_tile<Partition_Size>, Key key, Val val)
    {
        Val o;
        bool f;
        return run(pg::POP_INSERT_DELETE, key, val, o, f);
    }
    __device__ bool insert_with_delete(cooperative_groups::thread_block_tile<Partition_Size> tile, Key key)
    {
        return insert_with_delete(tile, key, Val(0));
    }
    __device__ bool insert_if_not_exists(cooperative_groups::thread_block_tile<Partition_Size>, Key key, Val val,
                                         Val &ext_val, bool &found)
    {
        Val o = 0;
        const bool r = run(pg::POP_INSERT_IF_NOT_EXISTS, key, val, o, found);
        if (r && found) ext_val = o;
        return r;
    }
    __device__ bool insert_if_not_exists_delete(cooperative_groups::thread_block_tile<Partition_Size>, Key key,
                                                Val val, Val &ext_val, bool &found)
    {
        Val o = 0;
        const bool r = run(pg::POP_INSERT_IF_NOT_EXISTS_DELETE, key, val, o, found);
        if (r && found) ext_val = o;
        return r;
    }
    __device__ bool query(cooperative_groups::thread_block_tile<Partition_Size>, Key key, Val &val)
    {
        Val o = 0;
        bool f;
        const bool r = run(pg::POP_QUERY, key, Val(0), o, f);
        if (r) val = o;
        return r;
    }
    __device__ bool remove(cooperative_groups::thread_block_tile<Partition_Size>, Key key)
    {
        Val o;
        bool f;
        return run(pg::POP_REMOVE, key, Val(0), o, f);
    }

    __device__ __inline__ cooperative_groups::thread_block_tile<Partition_Size> get_my_tile()
    {
        return cooperative_groups::tiled_partition<Partition_Size>(cooperative_groups::this_thread_block());
    }
    __host__ static uint64_t get_block_size(uint64_t) { return 1024; }
    __host__ static uint64_t get_num_blocks(uint64_t n) { return (Partition_Size * n - 1) / get_block_size(n) + 1; }
    __host__ uint64_t host_bytes_in_use() { return pg_table_bytes(host_handle(this)); }
    // bucketed_table::get_local_num_buckets / get_local_num_slots / get_num_slots
    // (bucketed_table.cuh:444-486): buckets and slots of the primary level, and
    // slots of every level
    __host__ uint64_t get_local_num_buckets()
    {
        pg_level_info li{};
        return pg_table_level_info(host_handle(this), 0, &li) == PG_OK ? li.nbuckets : 0;
    }
    __host__ uint64_t get_local_num_slots() { return get_local_num_buckets() * Bucket_Size; }
    __host__ uint64_t get_num_slots()
    {
        uint64_t total = 0;
        for (uint32_t l = 0; l < (Is_Recursive ? 2u : 1u); l++) {
            pg_level_info li{};
            if (pg_table_level_info(host_handle(this), l, &li) == PG_OK) total += li.nslots;
        }
        return total;
    }
    // bucketed_table::get_fill (:498-548): live slots of every level
    __host__ uint64_t get_fill()
    {
        pg_table *h = host_handle(this);
        uint64_t *d = nullptr;
        if (cudaMalloc(&d, 2 * sizeof(uint64_t)) != cudaSuccess) return 0;
        uint64_t total = 0;
        for (uint32_t l = 0; l < (Is_Recursive ? 2u : 1u); l++) {
            uint64_t hc[2] = {0, 0};
            cudaMemset(d, 0, 2 * sizeof(uint64_t));
            pg_table_count_fill(h, l, d, nullptr);
            cudaMemcpy(hc, d, sizeof(hc), cudaMemcpyDeviceToHost);
            total += hc[0] - hc[1];
        }
        cudaFree(d);
        return total;
    }
};

}  // namespace tables

namespace data_structs {
using tiny_static_table_4 =
    tables::static_table<uint64_t, uint16_t,
                         representations::dynamic_container<representations::key_val_pair, uint16_t>::representation, 4,
                         4, insert_schemes::bucket_insert, 20, probing_schemes::doubleHasher, hashers::murmurHasher>;
using tcf = tables::static_table<uint64_t, uint16_t,
                                 representations::dynamic_container<representations::key_val_pair, uint16_t>::representation,
                                 4, 16, insert_schemes::power_of_n_insert_shortcut_scheme, 2,
                                 probing_schemes::doubleHasher, hashers::murmurHasher, true, tiny_static_table_4>;
using hash_table_64 = tables::static_table<uint64_t, uint64_t, representations::key_val_pair, 4, 16,
                                           insert_schemes::bucket_insert, 20, probing_schemes::doubleHasher,
                                           hashers::murmurHasher>;
}  // namespace data_structs

}  // namespace poggers_b200
