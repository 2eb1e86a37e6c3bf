/*
 * poggers_oracle_bucketed.c -- CPU oracle for the reference's bucketed
 * two-choice filter with tombstone reuse (TEST INFRASTRUCTURE).
 *
 * Plain C restatement, one key at a time, of
 *   tables/bucketed_table.cuh:167-308          primary -> recursive backing dispatch
 *   insert_schemes/power_of_n_shortcut_buckets.cuh:141-740   two-choice shortcut scheme
 *   insert_schemes/linear_insert_buckets.cuh:110-420          linear backing scheme
 *   representations/packed_bucket.cuh:29-278                 bucket of packed slots
 *   representations/grouped_storage_sub_bits.cuh:36-255       grouped_bits_pair slot
 *   representations/dynamic_container.cuh:35-54              small-key tag
 * as instantiated by tests/src/delete_tests.cu:138-179 (del_TCF and
 * del_TCF_small).
 *
 * Slot: one little-endian word of 2*bits bits, tag in the low `bits` bits,
 * value in the high `bits` bits (join_in_storage, grouped_storage_sub_bits.cuh:75-93).
 * Empty word 0; tombstone word = tag all-ones, value 0 (get_tombstone is
 * Key{0}-1 clipped to the tag bits, atomic_reset writes value 0).  A key's tag
 * is the low `bits` bits of the raw key with 0 moved to 1 and all-ones moved
 * to all-ones - 1, so no key ever looks empty or deleted.
 *
 * In a bucket the reference's tile walks stripes of Partition_Size slots and
 * the lowest voting lane acts first, i.e. slots are visited in slot order for
 * every tile width; every CAS below succeeds in a sequential model because
 * the expected word is the one just read.
 *
 * Only tests/, __graft_entry__.smoke() and bench CPU legs use this file.
 */
#include "poggers_oracle.h"

#include <stdlib.h>
#include <string.h>

typedef struct blevel {
    pgo_level_cfg cfg;
    uint64_t nb;
    uint64_t seed;
    unsigned char *slots;
} blevel;

struct pgo_btable {
    pgo_bcfg cfg;
    uint32_t word_bytes;  /* 4 (16+16 bits) or 2 (8+8 bits) */
    uint32_t tag_mask;
    blevel lv[2];
};

static const uint64_t BPROBE_END = ~(uint64_t)0;

/* dynamic_container::get_smallKey over a `bits`-bit small key */
uint64_t pgo_btag(uint32_t bits, uint64_t key)
{
    const uint64_t mask = (bits == 8) ? 0xFFu : 0xFFFFu;
    uint64_t s = key & mask;
    if (s == 0) s += 1;
    if (s == mask) s -= 1;
    return s;
}

static inline uint64_t bhash(uint64_t key, uint64_t seed) { return pgo_murmur64a(&key, 8, seed); }

/* probe value i (< max_probes) of the level's probing scheme: XORPowerOfTwoHasher
 * (xor_power_of_two.cuh:64-89), linearProber (linear_probing.cuh:59-83),
 * doubleHasher (double_hashing.cuh:66-95) or powerOfTwoHasher (power_of_two.cuh:68-96);
 * rep_type::tag(key) is the small key (packed_bucket.cuh:214-218). */
typedef struct bprobe {
    uint32_t kind, max, i;
    uint64_t h1, h2, tag;
} bprobe;

static uint64_t bprobe_begin(bprobe *p, const blevel *L, uint64_t key, uint64_t tag)
{
    p->kind = L->cfg.probe;
    p->max = L->cfg.max_probes;
    p->i = 0;
    p->tag = tag;
    p->h1 = bhash(key, L->seed);
    p->h2 = (p->kind == PGO_PROBE_DOUBLE || p->kind == PGO_PROBE_P2) ? bhash(key, L->seed * L->seed) : 0;
    return p->h1;
}

static uint64_t bprobe_next(bprobe *p)
{
    p->i += 1;
    if (p->i >= p->max) return BPROBE_END;
    switch (p->kind) {
    case PGO_PROBE_DOUBLE: return p->h1 + (uint64_t)p->i * p->h2;
    case PGO_PROBE_LINEAR: return p->h1 + (uint64_t)p->i;
    case PGO_PROBE_P2: return p->h2;
    default: return p->h1 ^ (p->tag * 0x5bd1e995ULL);
    }
}

/* ---- slot words ---- */
static inline uint32_t wget(const pgo_btable *t, const blevel *L, uint64_t s)
{
    if (t->word_bytes == 4) { uint32_t w; memcpy(&w, L->slots + 4 * s, 4); return w; }
    uint16_t w; memcpy(&w, L->slots + 2 * s, 2); return w;
}
static inline void wset(const pgo_btable *t, blevel *L, uint64_t s, uint32_t w)
{
    if (t->word_bytes == 4) { memcpy(L->slots + 4 * s, &w, 4); return; }
    uint16_t h = (uint16_t)w; memcpy(L->slots + 2 * s, &h, 2);
}
static inline uint32_t bits_of(const pgo_btable *t) { return t->word_bytes * 4; }
static inline uint32_t wtag(const pgo_btable *t, uint32_t w) { return w & t->tag_mask; }
static inline uint32_t wval(const pgo_btable *t, uint32_t w) { return w >> bits_of(t); }
static inline uint32_t wjoin(const pgo_btable *t, uint64_t tag, uint64_t val)
{
    return (uint32_t)(tag & t->tag_mask) | ((uint32_t)(val & t->tag_mask) << bits_of(t));
}
static inline uint32_t wtomb(const pgo_btable *t) { return t->tag_mask; }

/* ---- packed_bucket.cuh ---- */
/* get_fill (:36-60): slots neither empty nor tombstone */
static int pb_fill(const pgo_btable *t, const blevel *L, uint64_t b)
{
    const uint32_t B = L->cfg.bucket_size;
    int f = 0;
    for (uint32_t i = 0; i < B; i++) {
        uint32_t g = wtag(t, wget(t, L, b * B + i));
        f += !(g == 0 || g == wtomb(t));
    }
    return f;
}
/* insert (:62-114): first empty slot, CAS(0 -> (tag, val)) */
static int pb_insert(pgo_btable *t, blevel *L, uint64_t b, uint64_t tag, uint64_t val)
{
    const uint32_t B = L->cfg.bucket_size;
    for (uint32_t i = 0; i < B; i++)
        if (wtag(t, wget(t, L, b * B + i)) == 0 && wget(t, L, b * B + i) == 0) {
            wset(t, L, b * B + i, wjoin(t, tag, val));
            return 1;
        }
    return 0;
}
/* insert_delete (:116-180): first empty or deleted slot; CAS from empty or
 * from the tombstone word */
static int pb_insert_delete(pgo_btable *t, blevel *L, uint64_t b, uint64_t tag, uint64_t val)
{
    const uint32_t B = L->cfg.bucket_size;
    for (uint32_t i = 0; i < B; i++) {
        uint32_t w = wget(t, L, b * B + i), g = wtag(t, w);
        if (g == 0 || g == wtomb(t)) {
            uint32_t expect = (g == 0) ? 0u : wtomb(t);
            if (w == expect) {
                wset(t, L, b * B + i, wjoin(t, tag, val));
                return 1;
            }
        }
    }
    return 0;
}
/* query (:182-212): first slot holding the tag, its value */
static int pb_query(const pgo_btable *t, const blevel *L, uint64_t b, uint64_t tag, uint64_t *val)
{
    const uint32_t B = L->cfg.bucket_size;
    for (uint32_t i = 0; i < B; i++) {
        uint32_t w = wget(t, L, b * B + i);
        if (wtag(t, w) == (tag & t->tag_mask)) {
            *val = wval(t, w);
            return 1;
        }
    }
    return 0;
}
/* remove (:220-264) + atomic_reset (grouped_storage_sub_bits.cuh:211-229):
 * first slot holding the tag, CAS((tag, val) -> tombstone word) */
static int pb_remove(pgo_btable *t, blevel *L, uint64_t b, uint64_t tag)
{
    const uint32_t B = L->cfg.bucket_size;
    for (uint32_t i = 0; i < B; i++) {
        uint32_t w = wget(t, L, b * B + i);
        if (wtag(t, w) == (tag & t->tag_mask)) {
            wset(t, L, b * B + i, wtomb(t));
            return 1;
        }
    }
    return 0;
}

#define BTC_MAX_PROBES 64

/* power_of_n_insert_shortcut_bucket_scheme insert / insert_with_delete
 * (power_of_n_shortcut_buckets.cuh:198-307, 309-419): a probed bucket whose
 * fill is below 3/4 of B takes the key at once; otherwise the buckets are
 * retried in increasing fill order, ties by probe order. */
static int tcb_place(pgo_btable *t, blevel *L, uint64_t key, uint64_t tag, uint64_t val, int with_delete)
{
    const int B = (int)L->cfg.bucket_size;
    uint64_t buckets[BTC_MAX_PROBES];
    int fill[BTC_MAX_PROBES];
    int n = 0, min_fill = B;
    bprobe p;
    for (uint64_t ps = bprobe_begin(&p, L, key, tag); ps != BPROBE_END && n < BTC_MAX_PROBES; ps = bprobe_next(&p)) {
        uint64_t b = ps % L->nb;
        buckets[n] = b;
        int cur = pb_fill(t, L, b);
        if (4 * cur < 3 * B) {
            if (with_delete ? pb_insert_delete(t, L, b, tag, val) : pb_insert(t, L, b, tag, val)) return 1;
            cur = B;
        }
        fill[n] = cur;
        if (cur < min_fill) min_fill = cur;
        n++;
    }
    int i = min_fill;
    while (i < B) {
        int next = B;
        for (int j = 0; j < n; j++) {
            if (fill[j] == i &&
                (with_delete ? pb_insert_delete(t, L, buckets[j], tag, val) : pb_insert(t, L, buckets[j], tag, val)))
                return 1;
            if (fill[j] > i && fill[j] < next) next = fill[j];
        }
        i = next;
    }
    return 0;
}

/* one level, one operation.  Returns the operation's boolean; *found and
 * *out as the reference's ext_val / found_val out-parameters. */
static int blevel_op(pgo_btable *t, blevel *L, int op, uint64_t key, uint64_t val, uint64_t *out, int *found)
{
    const uint64_t tag = pgo_btag(bits_of(t), key);
    const int linear = L->cfg.scheme == PGO_SCHEME_LINEAR_BUCKETED;
    const int B = (int)L->cfg.bucket_size;
    bprobe p;
    uint64_t ps;
    switch (op) {
    case PGO_BOP_INSERT:
    case PGO_BOP_INSERT_DELETE:
        if (!linear) return tcb_place(t, L, key, tag, val, op == PGO_BOP_INSERT_DELETE);
        /* linear_insert_buckets.cuh:192-236: the first probed bucket that takes it */
        for (ps = bprobe_begin(&p, L, key, tag); ps != BPROBE_END; ps = bprobe_next(&p)) {
            uint64_t b = ps % L->nb;
            if (op == PGO_BOP_INSERT_DELETE ? pb_insert_delete(t, L, b, tag, val) : pb_insert(t, L, b, tag, val))
                return 1;
        }
        return 0;
    case PGO_BOP_QUERY:
        /* query: shortcut scheme visits every probe (:676-707); the linear
         * scheme stops at the first bucket that is not full (:384-414) */
        for (ps = bprobe_begin(&p, L, key, tag); ps != BPROBE_END; ps = bprobe_next(&p)) {
            uint64_t b = ps % L->nb;
            if (pb_query(t, L, b, tag, out)) return 1;
            if (linear && pb_fill(t, L, b) != B) return 0;
        }
        return 0;
    case PGO_BOP_REMOVE:
        for (ps = bprobe_begin(&p, L, key, tag); ps != BPROBE_END; ps = bprobe_next(&p)) {
            uint64_t b = ps % L->nb;
            if (pb_remove(t, L, b, tag)) return 1;
            if (linear && pb_fill(t, L, b) != B) return 0;
        }
        return 0;
    default: /* PGO_BOP_INSERT_IF_NOT_EXISTS, PGO_BOP_INSERT_IF_NOT_EXISTS_DELETE */
    {
        const int del = op == PGO_BOP_INSERT_IF_NOT_EXISTS_DELETE;
        *found = 0;
        if (!linear) {
            /* :421-544, :546-674: query every probe first; a hit is reported
             * (and, for the _delete form, removed from that bucket) */
            for (ps = bprobe_begin(&p, L, key, tag); ps != BPROBE_END; ps = bprobe_next(&p)) {
                uint64_t b = ps % L->nb;
                if (pb_query(t, L, b, tag, out)) {
                    *found = 1;
                    if (del) pb_remove(t, L, b, tag);
                    return 1;
                }
            }
            return tcb_place(t, L, key, tag, val, del);
        }
        /* linear_insert_buckets.cuh:238-330: per probe, query then a plain insert */
        for (ps = bprobe_begin(&p, L, key, tag); ps != BPROBE_END; ps = bprobe_next(&p)) {
            uint64_t b = ps % L->nb;
            if (pb_query(t, L, b, tag, out)) {
                *found = 1;
                if (del) pb_remove(t, L, b, tag);
                return 1;
            }
            if (pb_insert(t, L, b, tag, val)) {
                *found = 0;
                return 1;
            }
        }
        return 0;
    }
    }
}

pgo_btable *pgo_btable_create(const pgo_bcfg *cfg, uint64_t seed)
{
    if (!cfg || (cfg->tag_bits != 16 && cfg->tag_bits != 8) || cfg->nlevels < 1 || cfg->nlevels > 2) return NULL;
    pgo_btable *t = (pgo_btable *)calloc(1, sizeof(pgo_btable));
    t->cfg = *cfg;
    t->word_bytes = cfg->tag_bits / 4;
    t->tag_mask = cfg->tag_bits == 16 ? 0xFFFFu : 0xFFu;
    uint64_t s = seed;
    for (uint32_t l = 0; l < cfg->nlevels; l++) {
        blevel *L = &t->lv[l];
        L->cfg = cfg->lv[l];
        if (L->cfg.nslots == 0 || L->cfg.bucket_size == 0 || L->cfg.max_probes == 0 ||
            (L->cfg.scheme != PGO_SCHEME_TWO_CHOICE_BUCKETED && L->cfg.scheme != PGO_SCHEME_LINEAR_BUCKETED)) {
            pgo_btable_destroy(t);
            return NULL;
        }
        L->nb = (L->cfg.nslots - 1) / L->cfg.bucket_size + 1;
        L->seed = s;  /* the recursive table gets seed*seed (bucketed_table.cuh:164) */
        L->slots = (unsigned char *)calloc(L->nb * L->cfg.bucket_size, t->word_bytes);
        if (!L->slots) {
            pgo_btable_destroy(t);
            return NULL;
        }
        s = s * s;
    }
    return t;
}

void pgo_btable_destroy(pgo_btable *t)
{
    if (!t) return;
    for (int l = 0; l < 2; l++) free(t->lv[l].slots);
    free(t);
}

uint64_t pgo_btable_level_bytes(const pgo_btable *t, int l)
{
    return t->lv[l].nb * t->lv[l].cfg.bucket_size * t->word_bytes;
}
uint64_t pgo_btable_level_nbuckets(const pgo_btable *t, int l) { return t->lv[l].nb; }
void *pgo_btable_level_data(pgo_btable *t, int l) { return t->lv[l].slots; }

/* bucketed_table dispatch (:167-308): the primary, then the backing table
 * when the primary reports failure */
int pgo_btable_op(pgo_btable *t, int op, uint64_t key, uint64_t val, uint64_t *out, int *found)
{
    uint64_t v = 0;
    int f = 0;
    int r = blevel_op(t, &t->lv[0], op, key, val, &v, &f);
    if (!r && t->cfg.nlevels > 1) {
        v = 0;
        f = 0;
        r = blevel_op(t, &t->lv[1], op, key, val, &v, &f);
    }
    if (out) *out = r ? v : 0;
    if (found) *found = f;
    return r;
}

uint64_t pgo_btable_bulk(pgo_btable *t, int op, const uint64_t *keys, const uint64_t *vals, uint64_t n,
                         uint64_t *out, uint8_t *ok, uint8_t *found)
{
    uint64_t c = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t v = 0;
        int f = 0;
        int r = pgo_btable_op(t, op, keys[i], vals ? vals[i] : 0, &v, &f);
        if (out) out[i] = v;
        if (ok) ok[i] = (uint8_t)r;
        if (found) found[i] = (uint8_t)f;
        c += (uint64_t)r;
    }
    return c;
}

/* get_fill (bucketed_table.cuh:498-548): live slots (neither empty nor deleted) */
uint64_t pgo_btable_count_fill(const pgo_btable *t, int l)
{
    uint64_t c = 0;
    const blevel *L = &t->lv[l];
    for (uint64_t b = 0; b < L->nb; b++) c += (uint64_t)pb_fill(t, L, b);
    return c;
}
