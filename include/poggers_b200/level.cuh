// level.cuh -- device-side bucket operations of one table level.
//
// A level is one insert scheme over its own bucket array: bucket_insert
// (include/poggers/insert_schemes/bucket_insert.cuh) or the two-choice
// shortcut scheme (include/poggers/insert_schemes/power_of_n_shortcut.cuh).
// A table is one level, or a primary level backed by a second one, exactly
// like the reference's static_table with a recursive backing table
// (include/poggers/tables/base_table.cuh:167-308).
//
// Layout in HBM (B = bucket size), bucket b at b * B * (sizeof K + sizeof V):
//   interleaved (default): B slots of {key, val}, the reference's own layout
//       (key_val_pair.cuh:72-74), so a value sits in the 32-byte sector of its
//       key: a hit needs no second DRAM access and an insert dirties one sector;
//   split: [ B keys | B vals ], keys contiguous (half the bytes per probe, but
//       a hit and an insert each touch a second sector).
// Random bucket reads are bound by DRAM transactions rather than bytes, which
// is why the interleaved layout is the default; both give identical results
// and dump to the same reference-layout bytes (pg_table_dump_level).
//
// One key is served by a group of G consecutive lanes (the reference's
// tile, `cg::thread_block_tile<Partition_Size>`), built on
// __ballot_sync / __shfl_sync / __reduce_add_sync with the group's own lane
// mask instead of cooperative-groups partitions.
//
// Semantics kept from the reference (sentinels included):
//   empty key 0, tombstone = empty - 1 (key_val_pair.cuh:70,115-117);
//   insert = CAS(empty -> key) on the first empty slot of a probed bucket in
//            slot order, then a plain val store (key_val_pair.cuh:84-95);
//   remove = CAS(key -> tombstone) on the first matching slot, val untouched;
//   bucket_insert query / remove stop at the first bucket holding an empty
//            slot (bucket_insert.cuh:283-285, 338-345);
//   two-choice query / remove visit every probed bucket, two-choice insert
//            takes a bucket whose fill is below 3/4 at once and otherwise the
//            least-filled bucket first (power_of_n_shortcut.cuh:327-435).
// Filled slots always form a prefix of each bucket (an insert only takes an
// empty slot after every earlier slot of its snapshot was seen filled, and
// nothing turns a filled slot back to empty), so the reference's per-stripe
// early exit equals "first match at or before the first empty slot", which
// is what is computed here for any group width G.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "hash.cuh"

namespace pg {

// FMT_KV64 / FMT_TAGVAL16 / FMT_TAG16 are the public formats (interleaved);
// the _SPLIT ids are the same formats with keys and values split per bucket.
// FMT_KV64_FP is FMT_KV64 with a fingerprint byte per slot (level_ops_fp).
enum fmt_kind : uint32_t {
    FMT_KV64 = 0,
    FMT_TAGVAL16 = 1,
    FMT_TAG16 = 2,
    FMT_KV64_SPLIT = 3,
    FMT_TAGVAL16_SPLIT = 4,
    FMT_KV64_FP = 5,
    FMT_PACKED16 = 6,  // bucketed filter, 16-bit tag + 16-bit value words (packed.cuh)
    FMT_PACKED8 = 7    // bucketed filter, 8-bit tag + 8-bit value words
};
enum scheme_kind : uint32_t { SCHEME_BUCKET = 0, SCHEME_TWO_CHOICE = 1 };

constexpr int kTwoChoiceMaxProbes = 4;
// Off by default: with the second read only when the first choice is at or
// above the shortcut threshold (inserts) or missed (queries), and the
// filters' kernels held to 40 registers, measured on B200 (G ops/s, insert +
// both queries): TCF 2^22 slots 22.1 -> 31.9, 2^28 14.6 -> 17.4, tag-only
// filter 2^28 20.5 -> 24.8.
#ifndef PG_TWO_CHOICE_PREFETCH
#define PG_TWO_CHOICE_PREFETCH 0
#endif
// read a two-choice key's second bucket together with its first (see insert_two_choice)
constexpr bool kTwoChoicePrefetch = PG_TWO_CHOICE_PREFETCH != 0;

struct level_desc {
    unsigned char *base;   // bucket array
    fastmod64 nbmod;       // d = number of buckets
    uint64_t seed, seed2;  // hasher seeds (s, s*s)
    uint32_t bucket_size, max_probes, scheme, probe;
    uint32_t bucket_bytes;
    uint32_t fp_resident;  // 1 when the fingerprint array fits in L2 and is kept there (evict-last loads)
    unsigned char *fp;     // FMT_KV64_FP: one fingerprint byte per slot, else null
};

struct table_desc {
    level_desc lv[2];
    uint32_t nlevels, format;
};

template <class Kt, class Vt, bool HasVal, bool Split, Kt Tomb, bool Tag>
struct fmt_base {
    using K = Kt;
    using V = Vt;
    static constexpr bool kHasVal = HasVal;
    static constexpr bool kSplit = Split && HasVal;
    static constexpr K kTomb = Tomb;
    // bytes between consecutive keys, and between consecutive values
    static constexpr uint32_t kKeyStride = (kSplit || !HasVal) ? (uint32_t)sizeof(K) : (uint32_t)(sizeof(K) + sizeof(V));
    static constexpr uint32_t kValStride = kSplit ? (uint32_t)sizeof(V) : kKeyStride;
    PG_HD static uint32_t val_offset(uint32_t B) { return kSplit ? B * (uint32_t)sizeof(K) : (uint32_t)sizeof(K); }
    PG_HD static K stored(uint64_t key)
    {
        if constexpr (Tag) return tag16(key);
        else return (K)key;
    }
    PG_HD static uint64_t tag(uint64_t key)
    {
        if constexpr (Tag) return tag16(key);
        else return key;
    }
};

template <int FMT> struct fmt_t;
// key_val_pair<uint64_t, uint64_t>: empty 0, tombstone ~0
template <> struct fmt_t<FMT_KV64> : fmt_base<unsigned long long, unsigned long long, true, false, ~0ULL, false> {};
template <> struct fmt_t<FMT_KV64_SPLIT> : fmt_base<unsigned long long, unsigned long long, true, true, ~0ULL, false> {};
template <> struct fmt_t<FMT_KV64_FP> : fmt_t<FMT_KV64> {};
// dynamic_container<key_val_pair, uint16_t>: 16-bit tag + 16-bit val, tombstone 0xFFFF
template <> struct fmt_t<FMT_TAGVAL16> : fmt_base<unsigned short, unsigned short, true, false, 0xFFFFu, true> {};
template <> struct fmt_t<FMT_TAGVAL16_SPLIT> : fmt_base<unsigned short, unsigned short, true, true, 0xFFFFu, true> {};
// dynamic_container<key_container, uint16_t>: tag only; queries report val 0
template <> struct fmt_t<FMT_TAG16> : fmt_base<unsigned short, unsigned short, false, false, 0xFFFFu, true> {};

// ---------------------------------------------------------------- groups
template <int G>
struct group {
    uint32_t gl;     // lane inside the group
    uint32_t gbase;  // warp lane of the group's lane 0
    uint32_t gmask;  // the group's lanes in the warp

    __device__ __forceinline__ static group make()
    {
        group g;
        uint32_t lane = threadIdx.x & 31u;
        g.gl = lane & (G - 1);
        g.gbase = lane - g.gl;
        g.gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << g.gbase);
        return g;
    }
    __device__ __forceinline__ uint32_t ballot(bool p) const
    {
        uint32_t b = __ballot_sync(gmask, p);
        return (G == 32) ? b : ((b >> gbase) & ((1u << G) - 1u));
    }
    template <class T>
    __device__ __forceinline__ T shfl(T v, uint32_t src_gl) const
    {
        if constexpr (sizeof(T) < 4) return (T)__shfl_sync(gmask, (unsigned)v, gbase + src_gl);
        else return __shfl_sync(gmask, v, gbase + src_gl);
    }
    __device__ __forceinline__ uint32_t sum(uint32_t v) const { return __reduce_add_sync(gmask, v); }
};

// One lane per key: every group operation is the lane's own value, so the
// bucket walk is straight-line thread-local code with no vote or shuffle.
template <>
struct group<1> {
    uint32_t gl, gbase, gmask;
    __device__ __forceinline__ static group make()
    {
        group g;
        g.gl = 0;
        g.gbase = threadIdx.x & 31u;
        g.gmask = 1u << g.gbase;
        return g;
    }
    __device__ __forceinline__ uint32_t ballot(bool p) const { return p ? 1u : 0u; }
    template <class T>
    __device__ __forceinline__ T shfl(T v, uint32_t) const { return v; }
    __device__ __forceinline__ uint32_t sum(uint32_t v) const { return v; }
};

// ---------------------------------------------------------------- loads
// L2-only loads (ld.global.cg): buckets are touched once per key, and a
// bucket another SM just updated by CAS must not be served from a stale L1.
// 32-byte global load (sm_100: ld.global with a 256-bit vector), L2 only.
__device__ __forceinline__ void ldcg32(const void *p, unsigned long long (&v)[4])
{
    asm volatile("ld.global.cg.v4.u64 {%0, %1, %2, %3}, [%4];"
                 : "=l"(v[0]), "=l"(v[1]), "=l"(v[2]), "=l"(v[3])
                 : "l"(p));
}

template <class K, int N>
__device__ __forceinline__ void load_keys(const K *p, K (&k)[N])
{
    constexpr int BYTES = N * (int)sizeof(K);
    if constexpr (BYTES >= 32 && BYTES % 32 == 0) {
        // a lane's span is a multiple of 32 bytes and starts on a 32-byte boundary
        // (bucket strides are multiples of the key span)
#pragma unroll
        for (int v = 0; v < BYTES / 32; ++v) {
            unsigned long long x[4];
            ldcg32(reinterpret_cast<const char *>(p) + 32 * v, x);
            memcpy(reinterpret_cast<char *>(k) + 32 * v, x, 32);
        }
    } else if constexpr (BYTES >= 16) {
        static_assert(BYTES % 16 == 0, "vector width");
#pragma unroll
        for (int v = 0; v < BYTES / 16; ++v) {
            uint4 x = __ldcg(reinterpret_cast<const uint4 *>(p) + v);
            memcpy(reinterpret_cast<char *>(k) + 16 * v, &x, 16);
        }
    } else if constexpr (BYTES == 8) {
        uint2 x = __ldcg(reinterpret_cast<const uint2 *>(p));
        memcpy(k, &x, 8);
    } else if constexpr (BYTES == 4) {
        unsigned int x = __ldcg(reinterpret_cast<const unsigned int *>(p));
        memcpy(k, &x, 4);
    } else {
        static_assert(BYTES == 2, "vector width");
        unsigned short x = __ldcg(reinterpret_cast<const unsigned short *>(p));
        memcpy(k, &x, 2);
    }
}

template <class K, int N>
__device__ __forceinline__ uint32_t eq_mask(const K (&k)[N], K v)
{
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) m |= (uint32_t)(k[i] == v) << i;
    return m;
}

// a[i] for a runtime i without indexing the register array
template <class T, int N>
__device__ __forceinline__ T pick(const T (&a)[N], int i)
{
    T r = a[0];
#pragma unroll
    for (int j = 1; j < N; ++j) r = (j == i) ? a[j] : r;
    return r;
}

template <class T>
__device__ __forceinline__ T ldcg_scalar(const T *p)
{
    return __ldcg(p);
}

// ---------------------------------------------------------------- level ops
// Compile-time bucket size B served by groups of G lanes.  Lane gl < ACT
// owns slots [gl*N, gl*N + N).
template <int FMT, int B, int G>
struct level_ops {
    using F = fmt_t<FMT>;
    using K = typename F::K;
    using V = typename F::V;
    static constexpr int ACT = B < G ? B : G;
    static constexpr int N = B < G ? 1 : B / G;
    static_assert(N <= 32, "slots per lane");

    __device__ __forceinline__ static unsigned char *bucket_of(const level_desc &L, uint64_t b)
    {
        return L.base + b * (uint64_t)L.bucket_bytes;
    }
    __device__ __forceinline__ static K *key_ptr(const level_desc &L, uint64_t b, int slot)
    {
        return reinterpret_cast<K *>(bucket_of(L, b) + slot * F::kKeyStride);
    }
    __device__ __forceinline__ static V *val_ptr(const level_desc &L, uint64_t b, int slot)
    {
        return reinterpret_cast<V *>(bucket_of(L, b) + F::val_offset(B) + slot * F::kValStride);
    }

    // A lane's view of its slots of one bucket: the keys, and with the
    // interleaved layout also the values (they arrive in the same load).
    struct snap {
        K k[N];
        V v[N];
    };
    static constexpr bool kValsInSnap = F::kHasVal && !F::kSplit;

    // Load this lane's slots of bucket b; lanes past the bucket hold no slot.
    __device__ __forceinline__ static void load(const level_desc &L, const group<G> &g, uint64_t b, snap &s,
                                                bool &active)
    {
        active = (int)g.gl < ACT;
        if (!active) {
#pragma unroll
            for (int i = 0; i < N; ++i) s.k[i] = F::kTomb;  // neither empty nor a stored key's slot
            return;
        }
        const K *p = key_ptr(L, b, (int)g.gl * N);
        if constexpr (kValsInSnap) {
            static_assert(sizeof(K) == sizeof(V), "interleaved slots pair equal-width key and value");
            K w[2 * N];
            load_keys<K, 2 * N>(p, w);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                s.k[i] = w[2 * i];
                s.v[i] = (V)w[2 * i + 1];
            }
        } else {
            load_keys<K, N>(p, s.k);
        }
    }

    // first slot (in slot order) whose lane-local bit is set, or -1
    __device__ __forceinline__ static int first(const group<G> &g, uint32_t m)
    {
        uint32_t bal = g.ballot(m != 0);
        if (!bal) return -1;
        uint32_t ln = __ffs(bal) - 1;
        int bit = g.shfl((int)__ffs(m) - 1, ln);
        return (int)ln * N + bit;
    }

    // CAS(empty -> sk) on the empty slots of the snapshot, in slot order.
    __device__ __forceinline__ static bool insert_into(const level_desc &L, const group<G> &g, uint64_t b, K sk,
                                                       V val, uint32_t emp)
    {
        while (true) {
            uint32_t bal = g.ballot(emp != 0);
            if (!bal) return false;
            uint32_t leader = __ffs(bal) - 1;
            bool ok = false;
            if (g.gl == leader) {
                int i = __ffs(emp) - 1;
                int slot = (int)g.gl * N + i;
                if (atomicCAS(key_ptr(L, b, slot), (K)0, sk) == (K)0) {
                    ok = true;
                    if constexpr (F::kHasVal) *val_ptr(L, b, slot) = val;
                } else {
                    emp &= emp - 1;
                }
            }
            if (g.ballot(ok)) return true;
        }
    }

    // CAS(sk -> tombstone) on the matching slots, in slot order.
    __device__ __forceinline__ static bool remove_from(const level_desc &L, const group<G> &g, uint64_t b, K sk,
                                                       uint32_t match)
    {
        while (true) {
            uint32_t bal = g.ballot(match != 0);
            if (!bal) return false;
            uint32_t leader = __ffs(bal) - 1;
            bool ok = false;
            if (g.gl == leader) {
                int i = __ffs(match) - 1;
                int slot = (int)g.gl * N + i;
                if (atomicCAS(key_ptr(L, b, slot), sk, F::kTomb) == sk) ok = true;
                else match &= match - 1;
            }
            if (g.ballot(ok)) return true;
        }
    }

    // value of `slot`: from the owning lane's snapshot (interleaved layout) or
    // one more load of the value (split layout)
    __device__ __forceinline__ static V read_val(const level_desc &L, const group<G> &g, uint64_t b, int slot,
                                                 const snap &s)
    {
        if constexpr (!F::kHasVal) {
            return (V)0;
        } else if constexpr (kValsInSnap) {
            return g.shfl(pick(s.v, slot % N), (uint32_t)(slot / N));
        } else {
            V v = 0;
            if ((int)g.gl == slot / N) v = ldcg_scalar(val_ptr(L, b, slot));
            return g.shfl(v, (uint32_t)(slot / N));
        }
    }

    __device__ __forceinline__ static void begin(const level_desc &L, uint64_t key, probe_seq &ps)
    {
        ps.begin(L.probe, key, F::tag(key), L.seed, L.seed2);
    }

    // ---- insert: bucket_insert (bucket_insert.cuh:127-203)
    __device__ static bool insert_bucket_scheme(const level_desc &L, const group<G> &g, uint64_t key, V val)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        begin(L, key, ps);
        for (uint32_t i = 0; i < L.max_probes; ++i) {
            uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            uint64_t b = L.nbmod.mod(raw);
            snap k;
            bool act;
            load(L, g, b, k, act);
            uint32_t emp = act ? eq_mask(k.k, (K)0) : 0u;
            if (insert_into(L, g, b, sk, val, emp)) return true;
        }
        return false;
    }

    // ---- insert: two-choice shortcut (power_of_n_shortcut.cuh:327-435).
    // Probe bookkeeping is unrolled over kTwoChoiceMaxProbes so it stays in
    // registers.  With kTwoChoicePrefetch both choices of the common 2-probe
    // case are fetched together (one round trip, two random sectors for every
    // key); without it the second choice is read only when the first is at or
    // above the shortcut threshold (a second round trip for those keys, one
    // sector fewer for the others).
    __device__ static bool insert_two_choice(const level_desc &L, const group<G> &g, uint64_t key, V val)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        begin(L, key, ps);
        constexpr int MP = kTwoChoiceMaxProbes;
        uint64_t bk[MP];
        int fill[MP];
        int np = 0, min_fill = B;
        snap k1;
        bool act1 = false, have1 = false;
        // Groups of several lanes serve two-choice levels below 2^18 slots
        // (pg_table_lanes): there both choices are read together, so a key's
        // two fills come from one moment.  With the second read deferred, a
        // 2^16-slot TCF with 1 % backing failed 209-217 keys at 0.9 load,
        // against none with both read together (the reference's build: ~100).
        constexpr bool kPrefetch = kTwoChoicePrefetch || G > 1;
        if (kPrefetch && L.max_probes >= 2 && ps.at(0) != kProbeEnd && ps.at(1) != kProbeEnd) {
            load(L, g, L.nbmod.mod(ps.at(1)), k1, act1);
            have1 = true;
        }
        bool stop = false;
#pragma unroll
        for (int i = 0; i < MP; ++i) {
            bk[i] = 0;
            fill[i] = B;
            if (stop || (uint32_t)i >= L.max_probes) continue;
            uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) {
                stop = true;
                continue;
            }
            uint64_t b = L.nbmod.mod(raw);
            snap k;
            bool act;
            if (i == 1 && have1) {
                k = k1;
                act = act1;
            } else {
                load(L, g, b, k, act);
            }
            uint32_t emp = act ? eq_mask(k.k, (K)0) : 0u;
            int f = (int)g.sum(act ? (uint32_t)(N - __popc(emp)) : 0u);
            bk[i] = b;
            if (4 * f < 3 * B) {
                if (insert_into(L, g, b, sk, val, emp)) return true;
                f = B;
            }
            fill[i] = f;
            if (f < min_fill) min_fill = f;
            np = i + 1;
        }
        int lvl = min_fill;
        while (lvl < B) {
            int next = B;
#pragma unroll
            for (int j = 0; j < MP; ++j) {
                if (j < np && fill[j] == lvl) {
                    snap k;
                    bool act;
                    load(L, g, bk[j], k, act);
                    uint32_t emp = act ? eq_mask(k.k, (K)0) : 0u;
                    if (insert_into(L, g, bk[j], sk, val, emp)) return true;
                }
                if (j < np && fill[j] > lvl && fill[j] < next) next = fill[j];
            }
            lvl = next;
        }
        return false;
    }

    template <int SCHEME>
    __device__ __forceinline__ static bool insert_s(const level_desc &L, const group<G> &g, uint64_t key, V val)
    {
        if constexpr (SCHEME == SCHEME_BUCKET) return insert_bucket_scheme(L, g, key, val);
        else return insert_two_choice(L, g, key, val);
    }
    __device__ __forceinline__ static bool insert(const level_desc &L, const group<G> &g, uint64_t key, V val)
    {
        return L.scheme == SCHEME_BUCKET ? insert_bucket_scheme(L, g, key, val) : insert_two_choice(L, g, key, val);
    }

    // ---- query: bucket_insert (bucket_insert.cuh:295-357)
    __device__ static bool query_bucket_scheme(const level_desc &L, const group<G> &g, uint64_t key, V &out)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        begin(L, key, ps);
        {
            for (uint32_t i = 0; i < L.max_probes; ++i) {
                uint64_t raw = ps.at(i);
                if (raw == kProbeEnd) break;
                uint64_t b = L.nbmod.mod(raw);
                snap k;
                bool act;
                load(L, g, b, k, act);
                int fm = first(g, act ? eq_mask(k.k, sk) : 0u);
                int fe = first(g, act ? eq_mask(k.k, (K)0) : 0u);
                if (fm >= 0 && (fe < 0 || fm <= fe)) {
                    out = read_val(L, g, b, fm, k);
                    return true;
                }
                if (fe >= 0) return false;
            }
            return false;
        }
    }

    // ---- query: two-choice (power_of_n_shortcut.cuh:193-232, 437-468): every
    // probed bucket, no early exit; the first two are fetched together
    __device__ static bool query_two_choice(const level_desc &L, const group<G> &g, uint64_t key, V &out)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        begin(L, key, ps);
        uint64_t r0 = ps.at(0);
        if (r0 == kProbeEnd) return false;
        uint64_t b0 = L.nbmod.mod(r0);
        snap k0, k1;
        bool a0, a1 = false;
        uint64_t b1 = 0;
        bool two = L.max_probes >= 2 && ps.at(1) != kProbeEnd;
        load(L, g, b0, k0, a0);
        // the first match in probe order answers: the second choice is read
        // with the first (kTwoChoicePrefetch) or only after the first missed
        if (kTwoChoicePrefetch && two) {
            b1 = L.nbmod.mod(ps.at(1));
            load(L, g, b1, k1, a1);
        }
        int fm = first(g, a0 ? eq_mask(k0.k, sk) : 0u);
        if (fm >= 0) {
            out = read_val(L, g, b0, fm, k0);
            return true;
        }
        if (!two) return false;
        if (!kTwoChoicePrefetch) {
            b1 = L.nbmod.mod(ps.at(1));
            load(L, g, b1, k1, a1);
        }
        fm = first(g, a1 ? eq_mask(k1.k, sk) : 0u);
        if (fm >= 0) {
            out = read_val(L, g, b1, fm, k1);
            return true;
        }
        for (uint32_t i = 2; i < L.max_probes; ++i) {
            uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            uint64_t b = L.nbmod.mod(raw);
            snap k;
            bool act;
            load(L, g, b, k, act);
            fm = first(g, act ? eq_mask(k.k, sk) : 0u);
            if (fm >= 0) {
                out = read_val(L, g, b, fm, k);
                return true;
            }
        }
        return false;
    }

    template <int SCHEME>
    __device__ __forceinline__ static bool query_s(const level_desc &L, const group<G> &g, uint64_t key, V &out)
    {
        if constexpr (SCHEME == SCHEME_BUCKET) return query_bucket_scheme(L, g, key, out);
        else return query_two_choice(L, g, key, out);
    }
    __device__ __forceinline__ static bool query(const level_desc &L, const group<G> &g, uint64_t key, V &out)
    {
        return L.scheme == SCHEME_BUCKET ? query_bucket_scheme(L, g, key, out) : query_two_choice(L, g, key, out);
    }

    // ---- remove: bucket_insert stops at a bucket holding an empty slot
    // (bucket_insert.cuh:205-293); two-choice visits every probe
    // (power_of_n_shortcut.cuh:263-325, 470-501)
    template <int SCHEME>
    __device__ static bool remove_s(const level_desc &L, const group<G> &g, uint64_t key)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        begin(L, key, ps);
        constexpr bool early = (SCHEME == SCHEME_BUCKET);
        for (uint32_t i = 0; i < L.max_probes; ++i) {
            uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            uint64_t b = L.nbmod.mod(raw);
            snap k;
            bool act;
            load(L, g, b, k, act);
            uint32_t match = act ? eq_mask(k.k, sk) : 0u;
            uint32_t emp = act ? (eq_mask(k.k, (K)0) & ~match) : 0u;
            if (remove_from(L, g, b, sk, match)) return true;
            if (early && g.ballot(emp != 0)) return false;
        }
        return false;
    }
    __device__ __forceinline__ static bool remove(const level_desc &L, const group<G> &g, uint64_t key)
    {
        return L.scheme == SCHEME_BUCKET ? remove_s<SCHEME_BUCKET>(L, g, key) : remove_s<SCHEME_TWO_CHOICE>(L, g, key);
    }
};

// Runtime bucket size (any B >= 1): the reference's own stripe walk, lane gl
// owns slots gl, gl+G, gl+2G, ...  Serves backing levels whose bucket size
// differs from the primary's.
template <int FMT, int G>
struct level_ops_dyn {
    using F = fmt_t<FMT>;
    using K = typename F::K;
    using V = typename F::V;

    __device__ __forceinline__ static K *key_ptr(const level_desc &L, uint64_t b, uint32_t s)
    {
        return reinterpret_cast<K *>(L.base + b * (uint64_t)L.bucket_bytes + s * F::kKeyStride);
    }
    __device__ __forceinline__ static V *val_ptr(const level_desc &L, uint64_t b, uint32_t s)
    {
        return reinterpret_cast<V *>(L.base + b * (uint64_t)L.bucket_bytes + F::val_offset(L.bucket_size) +
                                     s * F::kValStride);
    }
    __device__ __forceinline__ static K key_at(const level_desc &L, uint64_t b, uint32_t s)
    {
        return ldcg_scalar(key_ptr(L, b, s));
    }

    // first slot index in slot order satisfying pred, or -1
    template <class P>
    __device__ __forceinline__ static int first(const level_desc &L, const group<G> &g, uint64_t b, P pred)
    {
        const uint32_t B = L.bucket_size;
        for (uint32_t s0 = 0; s0 < B; s0 += G) {
            uint32_t s = s0 + g.gl;
            bool p = s < B && pred(key_at(L, b, s));
            uint32_t bal = g.ballot(p);
            if (bal) return (int)(s0 + __ffs(bal) - 1);
        }
        return -1;
    }

    __device__ static bool insert_bucket(const level_desc &L, const group<G> &g, uint64_t b, K sk, V val)
    {
        const uint32_t B = L.bucket_size;
        for (uint32_t s0 = 0; s0 < B; s0 += G) {
            uint32_t s = s0 + g.gl;
            bool e = s < B && key_at(L, b, s) == (K)0;
            uint32_t bal = g.ballot(e);
            while (bal) {
                uint32_t leader = __ffs(bal) - 1;
                bool ok = false;
                if (g.gl == leader && atomicCAS(key_ptr(L, b, s), (K)0, sk) == (K)0) {
                    ok = true;
                    if constexpr (F::kHasVal) *val_ptr(L, b, s) = val;
                }
                if (g.ballot(ok)) return true;
                bal &= bal - 1;
            }
        }
        return false;
    }

    __device__ static bool remove_bucket(const level_desc &L, const group<G> &g, uint64_t b, K sk)
    {
        const uint32_t B = L.bucket_size;
        for (uint32_t s0 = 0; s0 < B; s0 += G) {
            uint32_t s = s0 + g.gl;
            bool m = s < B && key_at(L, b, s) == sk;
            uint32_t bal = g.ballot(m);
            while (bal) {
                uint32_t leader = __ffs(bal) - 1;
                bool ok = false;
                if (g.gl == leader && atomicCAS(key_ptr(L, b, s), sk, F::kTomb) == sk) ok = true;
                if (g.ballot(ok)) return true;
                bal &= bal - 1;
            }
        }
        return false;
    }

    __device__ static V read_val(const level_desc &L, uint64_t b, int slot)
    {
        if constexpr (!F::kHasVal) return (V)0;
        else return ldcg_scalar(val_ptr(L, b, slot));
    }

    __device__ static int fill_of(const level_desc &L, const group<G> &g, uint64_t b)
    {
        const uint32_t B = L.bucket_size;
        uint32_t c = 0;
        for (uint32_t s = g.gl; s < B; s += G) c += key_at(L, b, s) != (K)0;
        return (int)g.sum(c);
    }

    __device__ static bool insert(const level_desc &L, const group<G> &g, uint64_t key, V val)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        ps.begin(L.probe, key, F::tag(key), L.seed, L.seed2);
        if (L.scheme == SCHEME_BUCKET) {
            for (uint32_t i = 0; i < L.max_probes; ++i) {
                uint64_t raw = ps.at(i);
                if (raw == kProbeEnd) break;
                if (insert_bucket(L, g, L.nbmod.mod(raw), sk, val)) return true;
            }
            return false;
        }
        const int B = (int)L.bucket_size;
        uint64_t bk[kTwoChoiceMaxProbes];
        int fill[kTwoChoiceMaxProbes];
        int np = 0, min_fill = B;
        const uint32_t mp = L.max_probes < (uint32_t)kTwoChoiceMaxProbes ? L.max_probes : kTwoChoiceMaxProbes;
        for (uint32_t i = 0; i < mp; ++i) {
            uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            uint64_t b = L.nbmod.mod(raw);
            int f = fill_of(L, g, b);
            bk[np] = b;
            if (4 * f < 3 * B) {
                if (insert_bucket(L, g, b, sk, val)) return true;
                f = B;
            }
            fill[np] = f;
            if (f < min_fill) min_fill = f;
            ++np;
        }
        int lvl = min_fill;
        while (lvl < B) {
            int next = B;
            for (int j = 0; j < np; ++j) {
                if (fill[j] == lvl && insert_bucket(L, g, bk[j], sk, val)) return true;
                if (fill[j] > lvl && fill[j] < next) next = fill[j];
            }
            lvl = next;
        }
        return false;
    }

    __device__ static bool query(const level_desc &L, const group<G> &g, uint64_t key, V &out)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        ps.begin(L.probe, key, F::tag(key), L.seed, L.seed2);
        const bool early = (L.scheme == SCHEME_BUCKET);
        for (uint32_t i = 0; i < L.max_probes; ++i) {
            uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            uint64_t b = L.nbmod.mod(raw);
            int fm = first(L, g, b, [sk](K k) { return k == sk; });
            int fe = early ? first(L, g, b, [](K k) { return k == (K)0; }) : -1;
            if (fm >= 0 && (fe < 0 || fm <= fe)) {
                out = read_val(L, b, fm);
                return true;
            }
            if (fe >= 0) return false;
        }
        return false;
    }

    __device__ static bool remove(const level_desc &L, const group<G> &g, uint64_t key)
    {
        const K sk = F::stored(key);
        probe_seq ps;
        ps.begin(L.probe, key, F::tag(key), L.seed, L.seed2);
        const bool early = (L.scheme == SCHEME_BUCKET);
        for (uint32_t i = 0; i < L.max_probes; ++i) {
            uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            uint64_t b = L.nbmod.mod(raw);
            if (remove_bucket(L, g, b, sk)) return true;
            if (early && first(L, g, b, [sk](K k) { return k == (K)0 && k != sk; }) >= 0) return false;
        }
        return false;
    }
};

// ---------------------------------------------------------------- fingerprint index
// uint64 tables can keep one fingerprint byte per slot in a separate array
// (1/16 of the slot bytes: 64 MB for 2^26 slots), read with an L2
// evict-last policy so it stays resident while the slots stream past with
// evict-first.  A probe then reads its bucket's fingerprints from L2 and goes
// to DRAM only for a slot whose fingerprint matches, reading that 16-byte slot
// (key and value together).  Random DRAM requests per op -- the limit of the
// plain walk -- drop from ~2.7 per query and ~2.3 per insert at 0.9 load to
// ~0.55 and ~0 (an insert only writes its slot).
//
// Fingerprint of a slot: 0 empty, 0xFF tombstone (or the key ~0, which the
// reference cannot tell from one), else 1..254 from the top byte of the
// key's first hash.  An insert claims its slot in the fingerprint array: a
// CAS on the (L2-resident) fingerprint word holding the bucket's first empty
// byte sets that byte to the key's fingerprint, and the winner then writes
// key and value with one 16-byte store.  The claim is the insert's
// linearisation point, as the key CAS is in the reference; slots are still
// taken first-empty in slot order, so filled slots stay a prefix of each
// bucket.  The bucket_insert decisions are unchanged: first empty slot for
// insert; first match at or before the first empty slot for query; first
// match, then stop at a bucket with an empty non-matching slot, for remove.
__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_normal()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// fingerprint loads: kept in L2 (evict-last) while the whole array fits there;
// a larger array would only crowd out the slot lines of the region in use
__device__ __forceinline__ uint64_t fp_policy(const level_desc &L)
{
    return L.fp_resident ? l2_policy_evict_last() : l2_policy_evict_normal();
}
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

PG_HD uint8_t fp_of(uint64_t key, uint64_t h1)
{
    if (key == 0) return 0;
    if (key == ~0ULL) return 0xFF;
    uint8_t f = (uint8_t)(h1 >> 56);
    f += (f == 0);
    f -= (f == 0xFF);
    return f;
}

// bit i set when byte i of w equals f
__device__ __forceinline__ uint32_t bytes_eq4(uint32_t w, uint32_t f)
{
    const uint32_t r = __vcmpeq4(w, f * 0x01010101u);
    return ((r >> 7) & 1u) | ((r >> 14) & 2u) | ((r >> 21) & 4u) | ((r >> 28) & 8u);
}

template <int B>
struct level_ops_fp {
    static_assert(B == 4 || B == 8 || B == 16 || B == 32, "bucket size");
    using F = fmt_t<FMT_KV64>;
    using K = unsigned long long;
    using V = unsigned long long;
    static constexpr int NW = B / 4;  // fingerprint words per bucket

    __device__ __forceinline__ static void load_fp(const level_desc &L, uint64_t b, uint32_t (&w)[NW], uint64_t pol)
    {
        const unsigned char *p = L.fp + b * B;
        if constexpr (B == 4) {
            asm volatile("ld.global.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(w[0]) : "l"(p), "l"(pol));
        } else if constexpr (B == 8) {
            unsigned long long x;
            asm volatile("ld.global.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(x) : "l"(p), "l"(pol));
            w[0] = (uint32_t)x;
            w[1] = (uint32_t)(x >> 32);
        } else {
#pragma unroll
            for (int q = 0; q < B / 16; ++q) {
                unsigned long long x, y;
                asm volatile("ld.global.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
                             : "=l"(x), "=l"(y)
                             : "l"(p + 16 * q), "l"(pol));
                w[4 * q + 0] = (uint32_t)x;
                w[4 * q + 1] = (uint32_t)(x >> 32);
                w[4 * q + 2] = (uint32_t)y;
                w[4 * q + 3] = (uint32_t)(y >> 32);
            }
        }
    }
    __device__ __forceinline__ static uint32_t match(const uint32_t (&w)[NW], uint32_t f)
    {
        uint32_t m = 0;
#pragma unroll
        for (int i = 0; i < NW; ++i) m |= bytes_eq4(w[i], f) << (4 * i);
        return m;
    }
    __device__ __forceinline__ static unsigned long long *slot_key(const level_desc &L, uint64_t b, int s)
    {
        return reinterpret_cast<unsigned long long *>(L.base + b * (uint64_t)L.bucket_bytes + 16 * s);
    }
    __device__ __forceinline__ static void load_slot(const level_desc &L, uint64_t b, int s, K &k, V &v, uint64_t pol)
    {
        asm volatile("ld.global.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
                     : "=l"(k), "=l"(v)
                     : "l"(slot_key(L, b, s)), "l"(pol));
    }
    __device__ __forceinline__ static void set_fp(const level_desc &L, uint64_t b, int s, uint32_t f)
    {
        // the slot's byte was 0 (insert) or a key's fingerprint (remove -> 0xFF): OR is exact
        if (!f) return;
        const uint64_t byte = b * B + s;
        unsigned int *w = reinterpret_cast<unsigned int *>(L.fp + (byte & ~3ULL));
        atomicOr(w, f << (8 * (byte & 3)));
    }
    // Claim the first empty slot of bucket b (slot order) by setting its
    // fingerprint byte to f; w is a snapshot of the bucket's fingerprints
    // (a snapshot is never fuller than the array, fill only grows).  Returns
    // the slot, or -1 when the bucket is full.  A failed CAS retries on the
    // word it returned; every failure means a byte of the word changed (0 ->
    // fingerprint, or fingerprint -> 0xFF on a remove), at most 16 times per
    // word, so the bound of 64 attempts is never the one that ends the loop.
    __device__ __forceinline__ static int claim(const level_desc &L, uint64_t b, const uint32_t (&w)[NW], uint32_t f)
    {
        if constexpr (B == 4) {
            unsigned int *p = reinterpret_cast<unsigned int *>(L.fp + b * B);
            uint32_t old = w[0];
            for (int it = 0; it < 64; ++it) {
                const uint32_t e = bytes_eq4(old, 0);
                if (!e) return -1;
                const int s = __ffs(e) - 1;
                const uint32_t prev = atomicCAS(p, old, old | (f << (8 * s)));
                if (prev == old) return s;
                old = prev;
            }
            return -1;
        } else {
#pragma unroll
            for (int q = 0; q < B / 8; ++q) {
                unsigned long long *p = reinterpret_cast<unsigned long long *>(L.fp + b * B + 8 * q);
                unsigned long long old = (unsigned long long)w[2 * q] | ((unsigned long long)w[2 * q + 1] << 32);
                for (int it = 0; it < 64; ++it) {
                    const uint32_t e = bytes_eq4((uint32_t)old, 0) | (bytes_eq4((uint32_t)(old >> 32), 0) << 4);
                    if (!e) break;  // this word is full: the bucket's next word
                    const int s = __ffs(e) - 1;
                    const unsigned long long prev = atomicCAS(p, old, old | ((unsigned long long)f << (8 * s)));
                    if (prev == old) return 8 * q + s;
                    old = prev;
                }
            }
            return -1;
        }
    }
    // key and value of a claimed slot, one 16-byte store
    __device__ __forceinline__ static void store_slot(const level_desc &L, uint64_t b, int s, K k, V v)
    {
        asm volatile("st.global.v2.u64 [%0], {%1, %2};" ::"l"(slot_key(L, b, s)), "l"(k), "l"(v) : "memory");
    }
    __device__ __forceinline__ static uint32_t upto(uint32_t e)
    {
        // slots 0 .. first empty (inclusive); all slots when none is empty
        if (!e) return (B == 32) ? 0xFFFFFFFFu : ((1u << B) - 1u);
        const uint32_t fe = __ffs(e) - 1;
        return (fe >= 31) ? 0xFFFFFFFFu : ((2u << fe) - 1u);
    }

    template <int SCHEME>
    __device__ static bool insert_s(const level_desc &L, const group<1> &, uint64_t key, V val)
    {
        static_assert(SCHEME == SCHEME_BUCKET, "fingerprints index bucket_insert levels");
        return insert_probes(L, key, val, 0, L.max_probes);
    }
    // The insert over probes [i0, i1) of the key's sequence: true when placed.
    // A bucket found full stays full (fill only grows during inserts), so a
    // caller may try probe 0 first and the rest later with the same result.
    __device__ __forceinline__ static bool insert_probes(const level_desc &L, uint64_t key, V val, uint32_t i0,
                                                         uint32_t i1)
    {
        probe_seq ps;
        ps.begin(L.probe, key, key, L.seed, L.seed2);
        const uint32_t f = fp_of(key, ps.h1);
        const uint64_t keep = fp_policy(L);
        for (uint32_t i = i0; i < i1 && i < L.max_probes; ++i) {
            const uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            const uint64_t b = L.nbmod.mod(raw);
            uint32_t w[NW];
            load_fp(L, b, w, keep);
            const int s = claim(L, b, w, f);
            if (s < 0) continue;
            if (f) {
                store_slot(L, b, s, key, val);
            } else {
                // the key 0 (the empty sentinel): as the reference's CAS of 0
                // over an empty key, it "succeeds" without filling the slot and
                // writes only the value
                slot_key(L, b, s)[1] = val;
            }
            return true;
        }
        return false;
    }

    template <int SCHEME>
    __device__ static bool query_s(const level_desc &L, const group<1> &, uint64_t key, V &out)
    {
        static_assert(SCHEME == SCHEME_BUCKET, "fingerprints index bucket_insert levels");
        probe_seq ps;
        ps.begin(L.probe, key, key, L.seed, L.seed2);
        const uint32_t f = fp_of(key, ps.h1);
        const uint64_t keep = fp_policy(L), stream = l2_policy_evict_first();
        for (uint32_t i = 0; i < L.max_probes; ++i) {
            const uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            const uint64_t b = L.nbmod.mod(raw);
            uint32_t w[NW];
            load_fp(L, b, w, keep);
            const uint32_t e = match(w, 0);
            uint32_t cand = match(w, f) & upto(e);
            while (cand) {
                const int s = __ffs(cand) - 1;
                K k;
                V v;
                load_slot(L, b, s, k, v, stream);
                if (k == (K)key) {
                    out = v;
                    return true;
                }
                cand &= cand - 1;
            }
            if (e) return false;
        }
        return false;
    }

    template <int SCHEME>
    __device__ static bool remove_s(const level_desc &L, const group<1> &, uint64_t key)
    {
        static_assert(SCHEME == SCHEME_BUCKET, "fingerprints index bucket_insert levels");
        probe_seq ps;
        ps.begin(L.probe, key, key, L.seed, L.seed2);
        const uint32_t f = fp_of(key, ps.h1);
        const uint64_t keep = fp_policy(L);
        for (uint32_t i = 0; i < L.max_probes; ++i) {
            const uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) break;
            const uint64_t b = L.nbmod.mod(raw);
            uint32_t w[NW];
            load_fp(L, b, w, keep);
            const uint32_t m = match(w, f);
            uint32_t cand = m;
            while (cand) {
                const int s = __ffs(cand) - 1;
                if (atomicCAS(slot_key(L, b, s), (K)key, F::kTomb) == (K)key) {
                    set_fp(L, b, s, 0xFFu);
                    return true;
                }
                cand &= cand - 1;
            }
            if (match(w, 0) & ~m) return false;
        }
        return false;
    }
};

// ---------------------------------------------------------------- table ops
// static_table dispatch: the primary level (compile-time bucket size B0 and
// scheme S0), then the backing level on failure or miss
// (base_table.cuh:167-187, 273-308).  The backing level is entered out of
// line so its registers do not weigh on the primary path.
template <int FMT, int G>
struct backing_ops {
    using F = fmt_t<FMT>;
    using V = typename F::V;
    using L1 = level_ops_dyn<FMT, G>;
    using L1x4 = level_ops<FMT, 4, G>;
    __device__ __noinline__ static bool insert(const level_desc L, const group<G> g, uint64_t key, V val)
    {
        if (L.bucket_size == 4 && G <= 4) return L1x4::insert(L, g, key, val);
        return L1::insert(L, g, key, val);
    }
    __device__ __noinline__ static bool query(const level_desc L, const group<G> g, uint64_t key, V *val)
    {
        V v = 0;
        bool r = (L.bucket_size == 4 && G <= 4) ? L1x4::query(L, g, key, v) : L1::query(L, g, key, v);
        *val = v;
        return r;
    }
    __device__ __noinline__ static bool remove(const level_desc L, const group<G> g, uint64_t key)
    {
        if (L.bucket_size == 4 && G <= 4) return L1x4::remove(L, g, key);
        return L1::remove(L, g, key);
    }
};

template <int FMT, int B, int G>
struct primary_ops {
    using type = level_ops<FMT, B, G>;
};
template <int B>
struct primary_ops<FMT_KV64_FP, B, 1> {
    using type = level_ops_fp<B>;
};

template <int FMT, int B0, int G, int S0, bool BK_ON = true>
struct table_ops {
    using F = fmt_t<FMT>;
    using V = typename F::V;
    using L0 = typename primary_ops<FMT, B0, G>::type;
    using BK = backing_ops<FMT == FMT_KV64_FP ? (int)FMT_KV64 : FMT, G>;

    __device__ __forceinline__ static bool insert(const table_desc &t, const group<G> &g, uint64_t key, V val)
    {
        if (L0::template insert_s<S0>(t.lv[0], g, key, val)) return true;
        if (!BK_ON || t.nlevels < 2) return false;
        return BK::insert(t.lv[1], g, key, val);
    }
    __device__ __forceinline__ static bool query(const table_desc &t, const group<G> &g, uint64_t key, V &val)
    {
        if (L0::template query_s<S0>(t.lv[0], g, key, val)) return true;
        if (!BK_ON || t.nlevels < 2) return false;
        return BK::query(t.lv[1], g, key, &val);
    }
    __device__ __forceinline__ static bool remove(const table_desc &t, const group<G> &g, uint64_t key)
    {
        if (L0::template remove_s<S0>(t.lv[0], g, key)) return true;
        if (!BK_ON || t.nlevels < 2) return false;
        return BK::remove(t.lv[1], g, key);
    }
};

}  // namespace pg
