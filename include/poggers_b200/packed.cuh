// packed.cuh -- device-side operations of the bucketed filter with tombstone
// reuse: buckets of packed (tag, value) words, a two-choice shortcut level
// backed by a linear-probing level.
//
// Reference: tables/bucketed_table.cuh:167-308 (primary -> backing dispatch),
// insert_schemes/power_of_n_shortcut_buckets.cuh:141-740 (two-choice shortcut
// scheme), insert_schemes/linear_insert_buckets.cuh:110-420 (linear scheme),
// representations/packed_bucket.cuh:29-278 (the bucket) and
// representations/grouped_storage_sub_bits.cuh:101-255 (grouped_bits_pair, the
// slot), as instantiated by tests/src/delete_tests.cu:138-179.
//
// Slot: one word of 2*W bits (W = 16: uint32, W = 8: uint16), the tag in the
// low W bits and the value in the high W bits; a bucket is B consecutive
// words, exactly the reference's device bytes.  Empty word 0, tombstone word
// = all-ones tag with value 0.  A key's tag is the low W bits of the raw key
// with 0 -> 1 and all-ones -> all-ones - 1 (dynamic_container.cuh:35-54).
// Every slot update is one CAS of the whole word, so a value is never seen
// without its tag (grouped_storage_sub_bits.cuh:126-229).
//
// The reference's tile walks a bucket in stripes and the lowest voting lane
// acts first, which is slot order for any tile width; here G lanes each load
// B/G consecutive words (one vector load), and "first in slot order" is the
// lowest lane's lowest bit.  Unlike bucket_insert, deletes leave holes, so no
// prefix rule applies: queries read the whole bucket, as the reference does.
#pragma once
#include <stdint.h>
#include <type_traits>
#include "level.cuh"

namespace pg {

enum : uint32_t { SCHEME_TWO_CHOICE_BUCKETED = 2, SCHEME_LINEAR_BUCKETED = 3 };

// bucketed filter operations (bucketed_table.cuh:167-308)
enum packed_op : int {
    POP_INSERT = 0,
    POP_QUERY = 1,
    POP_REMOVE = 2,
    POP_INSERT_DELETE = 3,              // insert_with_delete: a tombstone may be reused
    POP_INSERT_IF_NOT_EXISTS = 4,
    POP_INSERT_IF_NOT_EXISTS_DELETE = 5  // a key found is removed instead
};

template <int W>
struct pk {
    static_assert(W == 16 || W == 8, "tag bits");
    using word = std::conditional_t<W == 16, unsigned int, unsigned short>;
    using V = std::conditional_t<W == 16, unsigned short, unsigned char>;
    static constexpr uint32_t kMask = (1u << W) - 1u;
    static constexpr word kTombWord = (word)kMask;

    PG_HD static uint64_t tag(uint64_t key)
    {
        uint64_t s = key & kMask;
        s += (s == 0);
        s -= (s == kMask);
        return s;
    }
    PG_HD static word join(uint64_t t, uint64_t v) { return (word)((t & kMask) | ((v & kMask) << W)); }
    PG_HD static uint32_t tag_of(word w) { return (uint32_t)w & kMask; }
    PG_HD static V val_of(word w) { return (V)((uint32_t)w >> W); }
};

// One packed level with compile-time bucket size B, served by G lanes.
template <int W, int B, int G>
struct packed_level {
    using P = pk<W>;
    using word = typename P::word;
    using V = typename P::V;
    static_assert(B >= G && B % G == 0, "lanes per bucket");
    static constexpr int N = B / G;  // words per lane
    static_assert(N <= 32, "slots per lane");

    // What an operation needs of one read of a bucket, as lane-local bit masks
    // over the lane's N words (bit i = word gl*N + i), so the words themselves
    // die right after the read: empty words, tombstone words, dead tags (empty
    // or deleted: not counted in the fill), words holding the key's tag, and
    // the first such word (a remove's expected value).
    struct snap {
        uint32_t empty, tomb, dead, match;
        word mword;
    };

    __device__ __forceinline__ static word *slot(const level_desc &L, uint64_t b, int s)
    {
        return reinterpret_cast<word *>(L.base + b * (uint64_t)L.bucket_bytes) + s;
    }
    __device__ __forceinline__ static void load(const level_desc &L, const group<G> &g, uint64_t b, uint32_t t,
                                                snap &s)
    {
        word w[N];
        load_keys<word, N>(slot(L, b, (int)g.gl * N), w);
        s.empty = s.tomb = s.dead = s.match = 0;
        s.mword = 0;
#pragma unroll
        for (int i = N - 1; i >= 0; --i) {
            const uint32_t tg = P::tag_of(w[i]);
            s.empty |= (uint32_t)(w[i] == (word)0) << i;
            s.tomb |= (uint32_t)(w[i] == P::kTombWord) << i;
            s.dead |= (uint32_t)(tg == 0u || tg == P::kMask) << i;
            if (tg == t) {
                s.match |= 1u << i;
                s.mword = w[i];  // descending loop: ends on the lowest match
            }
        }
    }
    // live slots of the bucket: neither an empty nor a deleted tag (packed_bucket.cuh:36-60)
    __device__ __forceinline__ static int fill(const group<G> &g, const snap &s)
    {
        const uint32_t all = (N == 32) ? 0xFFFFFFFFu : ((1u << N) - 1u);
        return (int)g.sum((uint32_t)__popc((~s.dead) & all));
    }
    // CAS(expected -> desired) on the marked slots, in slot order; true on the
    // first success.  expected: 0 for an empty word, the tombstone word for a
    // deleted one, for a match the word read (the first) or read again (later
    // candidates, after a CAS lost a race; skipped if the tag changed meanwhile).
    __device__ __forceinline__ static bool cas_first(const level_desc &L, const group<G> &g, uint64_t b,
                                                     const snap &s, uint32_t m, word desired, bool by_tag,
                                                     uint32_t t)
    {
        const int first_match = s.match ? __ffs(s.match) - 1 : -1;
        while (true) {
            const uint32_t bal = g.ballot(m != 0);
            if (!bal) return false;
            const uint32_t leader = __ffs(bal) - 1;
            bool ok = false;
            if (g.gl == leader) {
                const int i = __ffs(m) - 1;
                word *p = slot(L, b, (int)g.gl * N + i);
                bool go = true;
                word expect;
                if (!by_tag) {
                    expect = ((s.empty >> i) & 1u) ? (word)0 : P::kTombWord;
                } else if (i == first_match) {
                    expect = s.mword;
                } else {
                    expect = ldcg_scalar(p);
                    go = P::tag_of(expect) == t;
                }
                if (go && atomicCAS(p, expect, desired) == expect) ok = true;
                else m &= m - 1;
            }
            if (g.ballot(ok)) return true;
        }
    }
    // first slot holding the tag: its value (packed_bucket.cuh:182-212)
    __device__ __forceinline__ static bool query_in(const group<G> &g, const snap &s, V &out)
    {
        const uint32_t bal = g.ballot(s.match != 0);
        if (!bal) return false;
        const word w = g.shfl(s.mword, __ffs(bal) - 1);
        out = P::val_of(w);
        return true;
    }
    // insert (:62-114): an empty word; insert_delete (:116-180): an empty or a deleted word
    __device__ __forceinline__ static bool place_in(const level_desc &L, const group<G> &g, uint64_t b,
                                                    const snap &s, word nw, bool reuse)
    {
        return cas_first(L, g, b, s, reuse ? (s.empty | s.tomb) : s.empty, nw, false, 0);
    }
    // remove (:220-264): the first slot holding the tag becomes the tombstone word
    __device__ __forceinline__ static bool remove_in(const level_desc &L, const group<G> &g, uint64_t b,
                                                     const snap &s, uint32_t t)
    {
        return cas_first(L, g, b, s, s.match, P::kTombWord, true, t);
    }

    // ---------------------------------------------------------------- schemes
    // two-choice shortcut placement (power_of_n_shortcut_buckets.cuh:198-419):
    // a probed bucket with fill below 3/4 of B takes the key at once; if none
    // does, buckets are retried in increasing fill order, ties in probe order.
    __device__ static bool tc_place(const level_desc &L, const group<G> &g, probe_seq &ps, uint32_t t, word nw,
                                    bool reuse)
    {
        uint64_t bk[kTwoChoiceMaxProbes];
        int fl[kTwoChoiceMaxProbes];
        int min_fill = B;
        bool more = true;  // the sequence ends at max_probes or at the end sentinel
#pragma unroll
        for (int j = 0; j < kTwoChoiceMaxProbes; ++j) {
            fl[j] = B;
            bk[j] = 0;
            if (!more || (uint32_t)j >= L.max_probes) continue;
            const uint64_t raw = ps.at((uint32_t)j);
            if (raw == kProbeEnd) {
                more = false;
                continue;
            }
            bk[j] = L.nbmod.mod(raw);
            snap s;
            load(L, g, bk[j], t, s);
            int f = fill(g, s);
            if (4 * f < 3 * B) {
                if (place_in(L, g, bk[j], s, nw, reuse)) return true;
                f = B;
            }
            fl[j] = f;
            min_fill = f < min_fill ? f : min_fill;
        }
        int i = min_fill;
        while (i < B) {
            int next = B;
#pragma unroll
            for (int j = 0; j < kTwoChoiceMaxProbes; ++j) {
                if (fl[j] == i) {
                    snap s;
                    load(L, g, bk[j], t, s);
                    if (place_in(L, g, bk[j], s, nw, reuse)) return true;
                }
                if (fl[j] > i && fl[j] < next) next = fl[j];
            }
            i = next;
        }
        return false;
    }

    // One operation on this level.  Returns the reference scheme's boolean;
    // out / found are its ext_val / found_val.
    __device__ __forceinline__ static bool op(const level_desc &L, const group<G> &g, int opk, uint64_t key,
                                              uint64_t val, V &out,
                              bool &found)
    {
        const uint64_t t = P::tag(key);
        const word nw = P::join(t, val);
        const bool linear = L.scheme == SCHEME_LINEAR_BUCKETED;
        probe_seq ps;
        ps.begin(L.probe, key, t, L.seed, L.seed2);
        switch (opk) {
        case POP_INSERT:
        case POP_INSERT_DELETE: {
            const bool reuse = opk == POP_INSERT_DELETE;
            if (!linear) return tc_place(L, g, ps, (uint32_t)t, nw, reuse);
            // linear_insert_buckets.cuh:192-236: the first probed bucket that takes it
            for (uint32_t i = 0; i < L.max_probes; ++i) {
                const uint64_t raw = ps.at(i);
                if (raw == kProbeEnd) break;
                const uint64_t b = L.nbmod.mod(raw);
                snap s;
                load(L, g, b, (uint32_t)t, s);
                if (place_in(L, g, b, s, nw, reuse)) return true;
            }
            return false;
        }
        case POP_QUERY:
        case POP_REMOVE: {
            // the shortcut scheme visits every probe (:676-740); the linear
            // scheme stops at the first bucket that is not full (:358-414)
            for (uint32_t i = 0; i < L.max_probes; ++i) {
                const uint64_t raw = ps.at(i);
                if (raw == kProbeEnd) break;
                const uint64_t b = L.nbmod.mod(raw);
                snap s;
                load(L, g, b, (uint32_t)t, s);
                if (opk == POP_QUERY) {
                    if (query_in(g, s, out)) return true;
                } else {
                    if (remove_in(L, g, b, s, (uint32_t)t)) return true;
                }
                if (linear && fill(g, s) != B) return false;
            }
            return false;
        }
        default: {
            // insert_if_not_exists[_delete]
            const bool del = opk == POP_INSERT_IF_NOT_EXISTS_DELETE;
            found = false;
            if (!linear) {
                // :421-674: every probe is queried first; a hit is reported and,
                // for the _delete form, removed from that bucket
                for (uint32_t i = 0; i < L.max_probes; ++i) {
                    const uint64_t raw = ps.at(i);
                    if (raw == kProbeEnd) break;
                    const uint64_t b = L.nbmod.mod(raw);
                    snap s;
                    load(L, g, b, (uint32_t)t, s);
                    if (query_in(g, s, out)) {
                        found = true;
                        if (del) remove_in(L, g, b, s, (uint32_t)t);
                        return true;
                    }
                }
                return tc_place(L, g, ps, (uint32_t)t, nw, del);
            }
            // linear_insert_buckets.cuh:238-330: per probe, query, then a plain insert
            for (uint32_t i = 0; i < L.max_probes; ++i) {
                const uint64_t raw = ps.at(i);
                if (raw == kProbeEnd) break;
                const uint64_t b = L.nbmod.mod(raw);
                snap s;
                load(L, g, b, (uint32_t)t, s);
                if (query_in(g, s, out)) {
                    found = true;
                    if (del) remove_in(L, g, b, s, (uint32_t)t);
                    return true;
                }
                if (place_in(L, g, b, s, nw, false)) return true;
            }
            return false;
        }
        }
    }
};

// primary level (bucket B0) and, when BK, the backing level (bucket B1):
// bucketed_table's dispatch, the backing table only when the primary fails.
template <int W, int B0, int B1, int G, bool BK>
struct packed_table {
    using V = typename pk<W>::V;
    __device__ __forceinline__ static bool op(const table_desc &t, const group<G> &g, int opk, uint64_t key,
                                              uint64_t val, V &out, bool &found)
    {
        out = 0;
        found = false;
        if (packed_level<W, B0, G>::op(t.lv[0], g, opk, key, val, out, found)) return true;
        if constexpr (BK) {
            if (t.nlevels > 1) {
                out = 0;
                found = false;
                return packed_level<W, B1, G>::op(t.lv[1], g, opk, key, val, out, found);
            }
        }
        return false;
    }
};

}  // namespace pg
