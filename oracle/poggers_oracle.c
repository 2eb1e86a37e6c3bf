/*
 * poggers_oracle.c -- CPU oracle for the POGGERS hot path (TEST INFRASTRUCTURE).
 *
 * Plain C11 restatement of the reference's table algorithms, one key at a
 * time, following the reference's own loop structure: a tile of Partition_Size
 * lanes walks each bucket in stripes of Partition_Size slots, votes, and lets
 * the lowest voting lane act first.  In a sequential model every lane's vote
 * and every compare-and-swap is resolved immediately, which is what the
 * reference's tile does when nothing else touches the table.
 *
 * Citations are paths inside the reference project (include/poggers/...).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this file.
 */
#define _GNU_SOURCE
#include "poggers_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------ */
/* MurmurHash64A: hash_schemes/murmurhash.cuh:20-61 (Austin Appleby's public
 * domain MurmurHash2, 64-bit variant A).  Keys are hashed as their 8 bytes in
 * host (little-endian) order: murmurHasher::hash copies the Key and hashes
 * sizeof(Key) bytes (murmurhash.cuh:93-100). */
uint64_t pgo_murmur64a(const void *key, int len, uint64_t seed)
{
    const uint64_t m = 0xc6a4a7935bd1e995ULL;
    const int r = 47;
    uint64_t h = seed ^ ((uint64_t)len * m);
    const unsigned char *p = (const unsigned char *)key;
    int nblocks = len / 8;
    for (int b = 0; b < nblocks; b++) {
        uint64_t k;
        memcpy(&k, p + 8 * b, 8);
        k *= m;
        k ^= k >> r;
        k *= m;
        h ^= k;
        h *= m;
    }
    const unsigned char *tail = p + 8 * nblocks;
    switch (len & 7) {
    case 7: h ^= (uint64_t)tail[6] << 48; /* fall through */
    case 6: h ^= (uint64_t)tail[5] << 40; /* fall through */
    case 5: h ^= (uint64_t)tail[4] << 32; /* fall through */
    case 4: h ^= (uint64_t)tail[3] << 24; /* fall through */
    case 3: h ^= (uint64_t)tail[2] << 16; /* fall through */
    case 2: h ^= (uint64_t)tail[1] << 8;  /* fall through */
    case 1: h ^= (uint64_t)tail[0]; h *= m;
    }
    h ^= h >> r;
    h *= m;
    h ^= h >> r;
    return h;
}

static inline uint64_t hash_key(uint64_t key, uint64_t seed)
{
    return pgo_murmur64a(&key, 8, seed);
}

/* internal_dynamic_container::get_smallKey, representations/dynamic_container.cuh:35-50:
 * the low 16 bits of the RAW key; 0 (empty) -> 1, 0xFFFF (tombstone) -> 0xFFFE. */
uint64_t pgo_tag16(uint64_t key)
{
    uint16_t s = (uint16_t)key;
    if (s == 0) s += 1;
    if (s == 0xFFFFu) s -= 1;
    return s;
}

/* rep_type::tag(key): key_val_pair::tag is the key itself (key_val_pair.cuh:127-131);
 * the dynamic container returns the small key (dynamic_container.cuh:52-54). */
static inline uint64_t rep_tag(uint32_t format, uint64_t key)
{
    return format == PGO_FMT_KV64 ? key : pgo_tag16(key);
}

/* ------------------------------------------------------------------------ */
/* Probing schemes.  begin() / next() / end() as in
 *   double_hashing.cuh:66-95   h1, h1+i*h2 with hashers seeded seed, seed*seed
 *   linear_probing.cuh:59-83   h, h+i
 *   power_of_two.cuh:68-96     h1, h2 (Max_probes == 2)
 *   xor_power_of_two.cuh:64-89 h1, h1 ^ (tag * 0x5bd1e995) (Max_probes == 2)
 * The caller's loop stops when a value equals end() == ~0 (bucket_insert.cuh:135). */
typedef struct probe_it {
    uint32_t kind, max;
    int i;
    uint64_t h1, h2, tag;
} probe_it;

static const uint64_t PROBE_END = ~(uint64_t)0;

static uint64_t probe_begin(probe_it *it, uint32_t kind, uint32_t max, uint64_t seed,
                            uint64_t key, uint64_t tag)
{
    it->kind = kind;
    it->max = max;
    it->i = 0;
    it->tag = tag;
    it->h1 = hash_key(key, seed);
    it->h2 = (kind == PGO_PROBE_DOUBLE || kind == PGO_PROBE_P2) ? hash_key(key, seed * seed) : 0;
    return it->h1;
}

static uint64_t probe_next(probe_it *it)
{
    it->i += 1;
    if ((uint32_t)it->i >= it->max) return PROBE_END;
    switch (it->kind) {
    case PGO_PROBE_DOUBLE: return it->h1 + (uint64_t)(int64_t)it->i * it->h2;
    case PGO_PROBE_LINEAR: return it->h1 + (uint64_t)(int64_t)it->i;
    case PGO_PROBE_P2: return it->h2;
    default: return it->h1 ^ (it->tag * 0x5bd1e995ULL);
    }
}

int pgo_probe_values(uint32_t probe, uint64_t seed, uint32_t format, uint64_t key,
                     uint32_t max_probes, uint64_t *out)
{
    probe_it it;
    int n = 0;
    for (uint64_t v = probe_begin(&it, probe, max_probes, seed, key, rep_tag(format, key));
         v != PROBE_END; v = probe_next(&it))
        out[n++] = v;
    return n;
}

/* ------------------------------------------------------------------------ */
/* Table model.  One level = one insert scheme over its own slot array
 * (each insert scheme's generate_on_device: min_buckets = (nslots-1)/B + 1,
 * zero-filled).  Level 1 is static_table's recursive backing table, created
 * with seed*seed (tables/base_table.cuh:122-125). */
typedef struct level {
    pgo_level_cfg cfg;
    uint64_t nb;
    uint64_t seed;
    unsigned char *slots;
} level;

struct pgo_table {
    pgo_cfg cfg;
    uint32_t slot_bytes;
    level lv[2];
};

static uint32_t fmt_slot_bytes(uint32_t f)
{
    return f == PGO_FMT_KV64 ? 16u : (f == PGO_FMT_TAGVAL16 ? 4u : 2u);
}

pgo_table *pgo_table_create(const pgo_cfg *cfg, uint64_t seed)
{
    if (!cfg || cfg->nlevels < 1 || cfg->nlevels > 2 || cfg->format > PGO_FMT_TAG16) return NULL;
    if (cfg->partition < 1 || cfg->partition > 32) return NULL;
    pgo_table *t = (pgo_table *)calloc(1, sizeof(pgo_table));
    t->cfg = *cfg;
    t->slot_bytes = fmt_slot_bytes(cfg->format);
    uint64_t s = seed;
    for (uint32_t l = 0; l < cfg->nlevels; l++) {
        level *L = &t->lv[l];
        L->cfg = cfg->lv[l];
        if (L->cfg.nslots == 0 || L->cfg.bucket_size == 0 || L->cfg.max_probes == 0) {
            pgo_table_destroy(t);
            return NULL;
        }
        L->nb = (L->cfg.nslots - 1) / L->cfg.bucket_size + 1;
        L->seed = s;
        L->slots = (unsigned char *)calloc(L->nb * L->cfg.bucket_size, t->slot_bytes);
        s = s * s;
    }
    return t;
}

void pgo_table_destroy(pgo_table *t)
{
    if (!t) return;
    for (int l = 0; l < 2; l++) free(t->lv[l].slots);
    free(t);
}

void pgo_table_clear(pgo_table *t)
{
    for (uint32_t l = 0; l < t->cfg.nlevels; l++)
        memset(t->lv[l].slots, 0, t->lv[l].nb * t->lv[l].cfg.bucket_size * t->slot_bytes);
}

uint64_t pgo_level_nbuckets(const pgo_table *t, int l) { return t->lv[l].nb; }
uint64_t pgo_level_bytes(const pgo_table *t, int l)
{
    return t->lv[l].nb * t->lv[l].cfg.bucket_size * t->slot_bytes;
}
void *pgo_level_data(pgo_table *t, int l) { return t->lv[l].slots; }
uint64_t pgo_level_seed(const pgo_table *t, int l) { return t->lv[l].seed; }

/* ---- slot accessors (reference AoS layout) ---- */
/* key_val_pair<Key,Val>: {Key key; Val val;} (key_val_pair.cuh:63-74);
 * key_container<Key,Val>: {Key key;} (key_only.cuh:24-34). */
static inline uint64_t slot_key(const pgo_table *t, const level *L, uint64_t s)
{
    const unsigned char *p = L->slots + s * t->slot_bytes;
    if (t->cfg.format == PGO_FMT_KV64) { uint64_t k; memcpy(&k, p, 8); return k; }
    uint16_t k; memcpy(&k, p, 2); return k;
}
static inline uint64_t slot_val(const pgo_table *t, const level *L, uint64_t s)
{
    const unsigned char *p = L->slots + s * t->slot_bytes;
    if (t->cfg.format == PGO_FMT_KV64) { uint64_t v; memcpy(&v, p + 8, 8); return v; }
    if (t->cfg.format == PGO_FMT_TAGVAL16) { uint16_t v; memcpy(&v, p + 2, 2); return v; }
    return 0; /* key_container::get_val returns 0 (key_only.cuh:75-77) */
}
static inline void slot_set(const pgo_table *t, level *L, uint64_t s, uint64_t k, uint64_t v, int write_val)
{
    unsigned char *p = L->slots + s * t->slot_bytes;
    if (t->cfg.format == PGO_FMT_KV64) {
        memcpy(p, &k, 8);
        if (write_val) memcpy(p + 8, &v, 8);
    } else {
        uint16_t k16 = (uint16_t)k;
        memcpy(p, &k16, 2);
        if (write_val && t->cfg.format == PGO_FMT_TAGVAL16) { uint16_t v16 = (uint16_t)v; memcpy(p + 2, &v16, 2); }
    }
}
/* stored form of a key: the key itself, or its 16-bit tag */
static inline uint64_t stored_key(const pgo_table *t, uint64_t key)
{
    return t->cfg.format == PGO_FMT_KV64 ? key : pgo_tag16(key);
}
/* tombstone = empty - 1 in the slot's key type (key_val_pair.cuh:115-117) */
static inline uint64_t tombstone(const pgo_table *t)
{
    return t->cfg.format == PGO_FMT_KV64 ? ~(uint64_t)0 : 0xFFFFu;
}

/* ------------------------------------------------------------------------ */
/* Sequential restatement.  P = Partition_Size; lane r of a stripe starting
 * at s0 owns slot s0 + r (the `for (i = rank; i < B; i += P)` loops). */

/* atomic_swap sequentially: CAS(empty -> stored key) succeeds iff the slot is
 * empty, then the (non-atomic) val store (key_val_pair.cuh:84-95). */
static int seq_swap(pgo_table *t, level *L, uint64_t s, uint64_t sk, uint64_t val)
{
    if (slot_key(t, L, s) != 0) return 0;
    slot_set(t, L, s, sk, val, 1);
    return 1;
}

/* atomic_reset: CAS(stored key -> tombstone), val untouched (key_val_pair.cuh:143-151) */
static int seq_reset(pgo_table *t, level *L, uint64_t s, uint64_t sk)
{
    if (slot_key(t, L, s) != sk) return 0;
    slot_set(t, L, s, tombstone(t), 0, 0);
    return 1;
}

/* bucket_insert::insert, insert_schemes/bucket_insert.cuh:127-203 */
static int bucket_insert_insert(pgo_table *t, level *L, uint64_t key, uint64_t val)
{
    const uint32_t B = L->cfg.bucket_size, P = t->cfg.partition;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END; ps = probe_next(&it)) {
        uint64_t base = (ps % L->nb) * B;
        for (uint32_t s0 = 0; s0 < B; s0 += P) {
            /* ballot: lanes whose slot is empty; leaders in lane order */
            for (uint32_t r = 0; r < P && s0 + r < B; r++) {
                if (slot_key(t, L, base + s0 + r) == 0 && seq_swap(t, L, base + s0 + r, sk, val)) return 1;
            }
        }
    }
    return 0;
}

/* bucket_insert::query, bucket_insert.cuh:295-357: per stripe, a match wins
 * (lowest lane's val); otherwise any empty slot in the stripe ends the search. */
static int bucket_insert_query(pgo_table *t, level *L, uint64_t key, uint64_t *val)
{
    const uint32_t B = L->cfg.bucket_size, P = t->cfg.partition;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END; ps = probe_next(&it)) {
        uint64_t base = (ps % L->nb) * B;
        for (uint32_t s0 = 0; s0 < B; s0 += P) {
            for (uint32_t r = 0; r < P && s0 + r < B; r++) {
                if (slot_key(t, L, base + s0 + r) == sk) {
                    *val = slot_val(t, L, base + s0 + r);
                    return 1;
                }
            }
            for (uint32_t r = 0; r < P && s0 + r < B; r++)
                if (slot_key(t, L, base + s0 + r) == 0) return 0;
        }
    }
    return 0;
}

/* bucket_insert::remove, bucket_insert.cuh:205-293: first match in stripe
 * order becomes a tombstone; a bucket that held an empty slot (and no match)
 * ends the search after the whole bucket was scanned. */
static int bucket_insert_remove(pgo_table *t, level *L, uint64_t key)
{
    const uint32_t B = L->cfg.bucket_size, P = t->cfg.partition;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END; ps = probe_next(&it)) {
        uint64_t base = (ps % L->nb) * B;
        int bucket_empty = 0;
        for (uint32_t s0 = 0; s0 < B; s0 += P) {
            for (uint32_t r = 0; r < P && s0 + r < B; r++) {
                uint64_t k = slot_key(t, L, base + s0 + r);
                if (k != sk && k == 0) bucket_empty = 1;
            }
            for (uint32_t r = 0; r < P && s0 + r < B; r++)
                if (slot_key(t, L, base + s0 + r) == sk && seq_reset(t, L, base + s0 + r, sk)) return 1;
        }
        if (bucket_empty) return 0;
    }
    return 0;
}

/* power_of_n_insert_shortcut_scheme::insert_into_bucket, power_of_n_shortcut.cuh:134-191 */
static int tc_insert_into_bucket(pgo_table *t, level *L, uint64_t bucket, uint64_t sk, uint64_t val)
{
    const uint32_t B = L->cfg.bucket_size, P = t->cfg.partition;
    uint64_t base = bucket * B;
    for (uint32_t s0 = 0; s0 < B; s0 += P)
        for (uint32_t r = 0; r < P && s0 + r < B; r++)
            if (slot_key(t, L, base + s0 + r) == 0 && seq_swap(t, L, base + s0 + r, sk, val)) return 1;
    return 0;
}

/* check_fill_bucket, power_of_n_shortcut.cuh:234-261: slots that are not empty */
static int tc_fill(pgo_table *t, level *L, uint64_t bucket)
{
    const uint32_t B = L->cfg.bucket_size;
    int fill = 0;
    for (uint32_t i = 0; i < B; i++) fill += slot_key(t, L, bucket * B + i) != 0;
    return fill;
}

#define TC_MAX_PROBES 64

/* power_of_n_insert_shortcut_scheme::insert, power_of_n_shortcut.cuh:327-435 */
static int two_choice_insert(pgo_table *t, level *L, uint64_t key, uint64_t val)
{
    const int B = (int)L->cfg.bucket_size;
    const uint64_t sk = stored_key(t, key);
    uint64_t buckets[TC_MAX_PROBES];
    int fill[TC_MAX_PROBES];
    int nprobe = 0, min_fill = B;
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END && nprobe < TC_MAX_PROBES; ps = probe_next(&it)) {
        uint64_t b = ps % L->nb;
        buckets[nprobe] = b;
        int cur = tc_fill(t, L, b);
        /* `current_fill < Bucket_Size*.75` (:352): exact as 4*fill < 3*B */
        if (4 * cur < 3 * B) {
            if (tc_insert_into_bucket(t, L, b, sk, val)) return 1;
            cur = B;
        }
        fill[nprobe] = cur;
        if (cur < min_fill) min_fill = cur;
        nprobe++;
    }
    /* retry in increasing-fill order, ties by probe index (:380-422) */
    int i = min_fill;
    while (i < B) {
        int next = B;
        for (int j = 0; j < nprobe; j++) {
            if (fill[j] == i && tc_insert_into_bucket(t, L, buckets[j], sk, val)) return 1;
            if (fill[j] > i && fill[j] < next) next = fill[j];
        }
        i = next;
    }
    return 0;
}

/* query_into_bucket / query, power_of_n_shortcut.cuh:193-232, 437-468: first
 * match in stripe order in each probed bucket, no early exit on empties. */
static int two_choice_query(pgo_table *t, level *L, uint64_t key, uint64_t *val)
{
    const uint32_t B = L->cfg.bucket_size;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END; ps = probe_next(&it)) {
        uint64_t base = (ps % L->nb) * B;
        for (uint32_t i = 0; i < B; i++)
            if (slot_key(t, L, base + i) == sk) { *val = slot_val(t, L, base + i); return 1; }
    }
    return 0;
}

/* remove_from_bucket / remove, power_of_n_shortcut.cuh:263-325, 470-501 */
static int two_choice_remove(pgo_table *t, level *L, uint64_t key)
{
    const uint32_t B = L->cfg.bucket_size;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END; ps = probe_next(&it)) {
        uint64_t base = (ps % L->nb) * B;
        for (uint32_t i = 0; i < B; i++)
            if (slot_key(t, L, base + i) == sk && seq_reset(t, L, base + i, sk)) return 1;
    }
    return 0;
}

static int level_insert(pgo_table *t, level *L, uint64_t key, uint64_t val)
{
    return L->cfg.scheme == PGO_SCHEME_BUCKET ? bucket_insert_insert(t, L, key, val)
                                              : two_choice_insert(t, L, key, val);
}
static int level_query(pgo_table *t, level *L, uint64_t key, uint64_t *val)
{
    return L->cfg.scheme == PGO_SCHEME_BUCKET ? bucket_insert_query(t, L, key, val)
                                              : two_choice_query(t, L, key, val);
}
static int level_remove(pgo_table *t, level *L, uint64_t key)
{
    return L->cfg.scheme == PGO_SCHEME_BUCKET ? bucket_insert_remove(t, L, key)
                                              : two_choice_remove(t, L, key);
}

/* static_table::insert / query / remove: primary, then the recursive table
 * on failure or miss (tables/base_table.cuh:167-187, 273-308). */
int pgo_insert(pgo_table *t, uint64_t key, uint64_t val)
{
    for (uint32_t l = 0; l < t->cfg.nlevels; l++)
        if (level_insert(t, &t->lv[l], key, val)) return 1;
    return 0;
}
int pgo_query(pgo_table *t, uint64_t key, uint64_t *val)
{
    for (uint32_t l = 0; l < t->cfg.nlevels; l++)
        if (level_query(t, &t->lv[l], key, val)) return 1;
    return 0;
}
int pgo_remove(pgo_table *t, uint64_t key)
{
    for (uint32_t l = 0; l < t->cfg.nlevels; l++)
        if (level_remove(t, &t->lv[l], key)) return 1;
    return 0;
}

uint64_t pgo_bulk_insert(pgo_table *t, const uint64_t *keys, const uint64_t *vals, uint64_t n, uint8_t *ok)
{
    uint64_t fails = 0;
    for (uint64_t i = 0; i < n; i++) {
        int r = pgo_insert(t, keys[i], vals ? vals[i] : 0);
        if (ok) ok[i] = (uint8_t)r;
        fails += !r;
    }
    return fails;
}

uint64_t pgo_bulk_query(pgo_table *t, const uint64_t *keys, uint64_t n, uint64_t *vals, uint8_t *found)
{
    uint64_t hits = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t v = 0;
        int r = pgo_query(t, keys[i], &v);
        if (vals) vals[i] = r ? v : 0;
        if (found) found[i] = (uint8_t)r;
        hits += r;
    }
    return hits;
}

uint64_t pgo_bulk_remove(pgo_table *t, const uint64_t *keys, uint64_t n, uint8_t *ok)
{
    uint64_t hits = 0;
    for (uint64_t i = 0; i < n; i++) {
        int r = pgo_remove(t, keys[i]);
        if (ok) ok[i] = (uint8_t)r;
        hits += r;
    }
    return hits;
}

uint64_t pgo_count_fill(const pgo_table *t, int l)
{
    const level *L = &t->lv[l];
    uint64_t n = L->nb * L->cfg.bucket_size, c = 0;
    for (uint64_t s = 0; s < n; s++) c += slot_key(t, L, s) != 0;
    return c;
}

/* ------------------------------------------------------------------------ */
/* Multithreaded host port.  Same slot layout and semantics, with real
 * compare-and-swap on the slot key (GCC __atomic builtins) so concurrent
 * workers behave like concurrent tiles: a worker reads a bucket snapshot,
 * then tries the empty (or matching) slots of the snapshot in index order. */

static inline uint64_t at_key(const pgo_table *t, const level *L, uint64_t s)
{
    unsigned char *p = L->slots + s * t->slot_bytes;
    if (t->cfg.format == PGO_FMT_KV64) return __atomic_load_n((uint64_t *)p, __ATOMIC_RELAXED);
    return __atomic_load_n((uint16_t *)p, __ATOMIC_RELAXED);
}
static inline int at_cas(const pgo_table *t, level *L, uint64_t s, uint64_t expect, uint64_t want)
{
    unsigned char *p = L->slots + s * t->slot_bytes;
    if (t->cfg.format == PGO_FMT_KV64) {
        uint64_t e = expect;
        return __atomic_compare_exchange_n((uint64_t *)p, &e, want, 0, __ATOMIC_ACQ_REL, __ATOMIC_RELAXED);
    }
    uint16_t e = (uint16_t)expect;
    return __atomic_compare_exchange_n((uint16_t *)p, &e, (uint16_t)want, 0, __ATOMIC_ACQ_REL, __ATOMIC_RELAXED);
}
static inline void at_store_val(const pgo_table *t, level *L, uint64_t s, uint64_t v)
{
    unsigned char *p = L->slots + s * t->slot_bytes;
    if (t->cfg.format == PGO_FMT_KV64) __atomic_store_n((uint64_t *)(p + 8), v, __ATOMIC_RELAXED);
    else if (t->cfg.format == PGO_FMT_TAGVAL16) __atomic_store_n((uint16_t *)(p + 2), (uint16_t)v, __ATOMIC_RELAXED);
}
static inline uint64_t at_val(const pgo_table *t, const level *L, uint64_t s)
{
    unsigned char *p = L->slots + s * t->slot_bytes;
    if (t->cfg.format == PGO_FMT_KV64) return __atomic_load_n((uint64_t *)(p + 8), __ATOMIC_RELAXED);
    if (t->cfg.format == PGO_FMT_TAGVAL16) return __atomic_load_n((uint16_t *)(p + 2), __ATOMIC_RELAXED);
    return 0;
}

static int mt_try_bucket(pgo_table *t, level *L, uint64_t base, uint64_t sk, uint64_t val)
{
    const uint32_t B = L->cfg.bucket_size;
    for (uint32_t i = 0; i < B; i++) {
        if (at_key(t, L, base + i) == 0 && at_cas(t, L, base + i, 0, sk)) {
            at_store_val(t, L, base + i, val);
            return 1;
        }
    }
    return 0;
}

static int mt_level_insert(pgo_table *t, level *L, uint64_t key, uint64_t val)
{
    const uint32_t B = L->cfg.bucket_size;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    if (L->cfg.scheme == PGO_SCHEME_BUCKET) {
        for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
             ps != PROBE_END; ps = probe_next(&it))
            if (mt_try_bucket(t, L, (ps % L->nb) * B, sk, val)) return 1;
        return 0;
    }
    uint64_t buckets[TC_MAX_PROBES];
    int fill[TC_MAX_PROBES];
    int nprobe = 0, min_fill = (int)B;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END && nprobe < TC_MAX_PROBES; ps = probe_next(&it)) {
        uint64_t b = ps % L->nb;
        buckets[nprobe] = b;
        int cur = 0;
        for (uint32_t i = 0; i < B; i++) cur += at_key(t, L, b * B + i) != 0;
        if (4 * cur < 3 * (int)B) {
            if (mt_try_bucket(t, L, b * B, sk, val)) return 1;
            cur = (int)B;
        }
        fill[nprobe] = cur;
        if (cur < min_fill) min_fill = cur;
        nprobe++;
    }
    int i = min_fill;
    while (i < (int)B) {
        int next = (int)B;
        for (int j = 0; j < nprobe; j++) {
            if (fill[j] == i && mt_try_bucket(t, L, buckets[j] * B, sk, val)) return 1;
            if (fill[j] > i && fill[j] < next) next = fill[j];
        }
        i = next;
    }
    return 0;
}

static int mt_level_query(pgo_table *t, level *L, uint64_t key, uint64_t *val)
{
    const uint32_t B = L->cfg.bucket_size;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END; ps = probe_next(&it)) {
        uint64_t base = (ps % L->nb) * B;
        int empty = 0;
        for (uint32_t i = 0; i < B; i++) {
            uint64_t k = at_key(t, L, base + i);
            if (k == sk) { *val = at_val(t, L, base + i); return 1; }
            empty |= (k == 0);
        }
        /* filled slots form a prefix of every bucket, so for bucket_insert an
         * empty slot anywhere in the bucket ends the search exactly as the
         * reference's per-stripe rule does */
        if (L->cfg.scheme == PGO_SCHEME_BUCKET && empty) return 0;
    }
    return 0;
}

static int mt_level_remove(pgo_table *t, level *L, uint64_t key)
{
    const uint32_t B = L->cfg.bucket_size;
    const uint64_t sk = stored_key(t, key);
    probe_it it;
    for (uint64_t ps = probe_begin(&it, L->cfg.probe, L->cfg.max_probes, L->seed, key, rep_tag(t->cfg.format, key));
         ps != PROBE_END; ps = probe_next(&it)) {
        uint64_t base = (ps % L->nb) * B;
        int empty = 0;
        for (uint32_t i = 0; i < B; i++) {
            uint64_t k = at_key(t, L, base + i);
            if (k == sk && at_cas(t, L, base + i, sk, tombstone(t))) return 1;
            if (k != sk && k == 0) empty = 1;
        }
        if (L->cfg.scheme == PGO_SCHEME_BUCKET && empty) return 0;
    }
    return 0;
}

typedef struct mt_job {
    pgo_table *t;
    int op;
    const uint64_t *keys;
    const uint64_t *vals_in;
    uint64_t *vals_out;
    uint8_t *flags;
    uint64_t lo, hi;
    uint64_t count;
} mt_job;

static void *mt_worker(void *arg)
{
    mt_job *j = (mt_job *)arg;
    pgo_table *t = j->t;
    uint64_t c = 0;
    for (uint64_t i = j->lo; i < j->hi; i++) {
        uint64_t key = j->keys[i];
        int r = 0;
        if (j->op == 0) {
            uint64_t v = j->vals_in ? j->vals_in[i] : 0;
            for (uint32_t l = 0; l < t->cfg.nlevels && !r; l++) r = mt_level_insert(t, &t->lv[l], key, v);
            c += !r;
        } else if (j->op == 1) {
            uint64_t v = 0;
            for (uint32_t l = 0; l < t->cfg.nlevels && !r; l++) r = mt_level_query(t, &t->lv[l], key, &v);
            if (j->vals_out) j->vals_out[i] = r ? v : 0;
            c += r;
        } else {
            for (uint32_t l = 0; l < t->cfg.nlevels && !r; l++) r = mt_level_remove(t, &t->lv[l], key);
            c += r;
        }
        if (j->flags) j->flags[i] = (uint8_t)r;
    }
    j->count = c;
    return NULL;
}

int pgo_online_cores(void)
{
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static uint64_t mt_run(pgo_table *t, int op, const uint64_t *keys, const uint64_t *vin, uint64_t *vout,
                       uint8_t *flags, uint64_t n, int nthreads)
{
    if (nthreads <= 0) nthreads = pgo_online_cores();
    if ((uint64_t)nthreads > n) nthreads = n ? (int)n : 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    mt_job *jobs = (mt_job *)calloc(nthreads, sizeof(mt_job));
    for (int w = 0; w < nthreads; w++) {
        jobs[w].t = t;
        jobs[w].op = op;
        jobs[w].keys = keys;
        jobs[w].vals_in = vin;
        jobs[w].vals_out = vout;
        jobs[w].flags = flags;
        jobs[w].lo = n * w / nthreads;
        jobs[w].hi = n * (w + 1) / nthreads;
        pthread_create(&th[w], NULL, mt_worker, &jobs[w]);
    }
    uint64_t total = 0;
    for (int w = 0; w < nthreads; w++) {
        pthread_join(th[w], NULL);
        total += jobs[w].count;
    }
    free(th);
    free(jobs);
    return total;
}

uint64_t pgo_mt_bulk_insert(pgo_table *t, const uint64_t *keys, const uint64_t *vals, uint64_t n, uint8_t *ok, int nthreads)
{
    return mt_run(t, 0, keys, vals, NULL, ok, n, nthreads);
}
uint64_t pgo_mt_bulk_query(pgo_table *t, const uint64_t *keys, uint64_t n, uint64_t *vals, uint8_t *found, int nthreads)
{
    return mt_run(t, 1, keys, NULL, vals, found, n, nthreads);
}
uint64_t pgo_mt_bulk_remove(pgo_table *t, const uint64_t *keys, uint64_t n, uint8_t *ok, int nthreads)
{
    return mt_run(t, 2, keys, NULL, NULL, ok, n, nthreads);
}

/* ------------------------------------------------------------------------ */
/* splitmix64 (Steele, Lea, Flood 2014): a bijection of its 64-bit state, so
 * distinct stream positions give distinct keys. */
void pgo_splitmix64_fill(uint64_t seed, uint64_t start, uint64_t n, uint64_t *out)
{
    for (uint64_t i = 0; i < n; i++) {
        uint64_t z = seed + (start + i + 1) * 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        out[i] = z ^ (z >> 31);
    }
}

/* ------------------------------------------------------------------------ */
/* Slab allocator model (one_size_slab_allocator, allocators/slab_one_size.cuh):
 * a pool of ceil(num_allocs / 4096) * 4096 objects; malloc returns a free
 * object or fails when none is left; free returns an object, and a free of an
 * object that is already free is a double free (offset_slab.cuh:473-478).
 * Sequential and deterministic (lowest free offset first): object identities
 * differ from a concurrent allocator's, but every count must agree. */
struct pgo_slab {
    uint64_t capacity;
    uint64_t nfree;
    uint64_t *bits; /* 1 = free */
};

pgo_slab *pgo_slab_create(uint64_t num_allocs)
{
    if (num_allocs == 0) return NULL;
    pgo_slab *s = (pgo_slab *)calloc(1, sizeof(pgo_slab));
    s->capacity = ((num_allocs - 1) / 4096 + 1) * 4096;
    s->nfree = s->capacity;
    s->bits = (uint64_t *)malloc(s->capacity / 8);
    memset(s->bits, 0xFF, s->capacity / 8);
    return s;
}

void pgo_slab_destroy(pgo_slab *s)
{
    if (!s) return;
    free(s->bits);
    free(s);
}

uint64_t pgo_slab_capacity(const pgo_slab *s) { return s->capacity; }
uint64_t pgo_slab_free_objects(const pgo_slab *s) { return s->nfree; }

/* offsets[i] = object offset or ~0; returns failures */
uint64_t pgo_slab_malloc(pgo_slab *s, uint64_t n, uint64_t *offsets)
{
    uint64_t fails = 0, w = 0;
    for (uint64_t i = 0; i < n; i++) {
        while (w < s->capacity / 64 && s->bits[w] == 0) w++;
        if (w == s->capacity / 64) {
            offsets[i] = ~(uint64_t)0;
            fails++;
            continue;
        }
        int b = __builtin_ctzll(s->bits[w]);
        s->bits[w] &= s->bits[w] - 1;
        s->nfree--;
        offsets[i] = w * 64 + (uint64_t)b;
    }
    return fails;
}

/* returns the number of rejected frees (double frees, offsets out of range) */
uint64_t pgo_slab_free(pgo_slab *s, uint64_t n, const uint64_t *offsets)
{
    uint64_t bad = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t o = offsets[i];
        if (o >= s->capacity) { bad++; continue; }
        uint64_t m = 1ULL << (o % 64);
        if (s->bits[o / 64] & m) { bad++; continue; }
        s->bits[o / 64] |= m;
        s->nfree++;
    }
    return bad;
}
