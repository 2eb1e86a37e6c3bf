/*
 * poggers_oracle.h -- CPU oracle for the POGGERS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms (hashing, probing, bucket_insert, power_of_n_insert_shortcut_scheme,
 * static_table fallback) used by the tests, by smoke() and by the CPU legs of
 * bench.py as the checker and the CPU baseline.  The product (poggers_b200)
 * never links or calls it.
 *
 * Tables are kept in the REFERENCE's slot layout (array-of-structs slots,
 * buckets of Bucket_Size consecutive slots), so a level's raw bytes compare
 * byte-for-byte with a dump of the reference's own device table.
 *
 * Parity pin: murmur and probe sequences are pinned against the reference's
 * own __host__ code compiled from its headers (oracle/ref_host_pin.cpp), and the
 * sequential table layout is pinned against golden dumps produced by the
 * reference's CUDA build (tests/golden/, generated by
 * tests/golden/make_golden.py).
 */
#ifndef POGGERS_ORACLE_H
#define POGGERS_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* slot formats (reference representations) */
enum {
    PGO_FMT_KV64 = 0,     /* key_val_pair<uint64_t,uint64_t>, 16 B slot */
    PGO_FMT_TAGVAL16 = 1, /* dynamic_container<key_val_pair,uint16_t> over <uint64,uint16>, 4 B slot */
    PGO_FMT_TAG16 = 2     /* dynamic_container<key_container,uint16_t>, 2 B slot (val reads 0) */
};

/* insert schemes */
enum {
    PGO_SCHEME_BUCKET = 0,     /* insert_schemes/bucket_insert.cuh */
    PGO_SCHEME_TWO_CHOICE = 1, /* insert_schemes/power_of_n_shortcut.cuh */
    PGO_SCHEME_TWO_CHOICE_BUCKETED = 2, /* insert_schemes/power_of_n_shortcut_buckets.cuh */
    PGO_SCHEME_LINEAR_BUCKETED = 3      /* insert_schemes/linear_insert_buckets.cuh */
};

/* probing schemes */
enum {
    PGO_PROBE_DOUBLE = 0,  /* probing_schemes/double_hashing.cuh */
    PGO_PROBE_LINEAR = 1,  /* probing_schemes/linear_probing.cuh */
    PGO_PROBE_P2 = 2,      /* probing_schemes/power_of_two.cuh */
    PGO_PROBE_XOR_P2 = 3   /* probing_schemes/xor_power_of_two.cuh */
};

typedef struct pgo_level_cfg {
    uint64_t nslots;
    uint32_t bucket_size;
    uint32_t max_probes;
    uint32_t scheme;
    uint32_t probe;
} pgo_level_cfg;

typedef struct pgo_cfg {
    uint32_t format;
    uint32_t partition;   /* reference Partition_Size (tile width), 1..32 */
    uint32_t nlevels;     /* 1 or 2 (primary + recursive backing table) */
    uint32_t pad;
    pgo_level_cfg lv[2];
} pgo_cfg;

typedef struct pgo_table pgo_table;

/* hashing / probing */
uint64_t pgo_murmur64a(const void *key, int len, uint64_t seed);
uint64_t pgo_tag16(uint64_t key);
/* Raw probe values (before % num_buckets) of `key` for a level hashed with `seed`.
 * Returns how many were written (< max_probes when the ~0 end sentinel is hit). */
int pgo_probe_values(uint32_t probe, uint64_t seed, uint32_t format, uint64_t key,
                     uint32_t max_probes, uint64_t *out);

/* table lifetime; level seeds follow static_table::generate_on_device:
 * level 0 gets `seed`, level 1 gets seed*seed. */
pgo_table *pgo_table_create(const pgo_cfg *cfg, uint64_t seed);
void pgo_table_destroy(pgo_table *t);
void pgo_table_clear(pgo_table *t);
uint64_t pgo_level_nbuckets(const pgo_table *t, int level);
uint64_t pgo_level_bytes(const pgo_table *t, int level);
void *pgo_level_data(pgo_table *t, int level);
uint64_t pgo_level_seed(const pgo_table *t, int level);

/* sequential single-key operations, one tile per key, in call order */
int pgo_insert(pgo_table *t, uint64_t key, uint64_t val);
int pgo_query(pgo_table *t, uint64_t key, uint64_t *val);
int pgo_remove(pgo_table *t, uint64_t key);

/* sequential bulk forms (batch order); any output pointer may be NULL */
uint64_t pgo_bulk_insert(pgo_table *t, const uint64_t *keys, const uint64_t *vals, uint64_t n, uint8_t *ok);
uint64_t pgo_bulk_query(pgo_table *t, const uint64_t *keys, uint64_t n, uint64_t *vals, uint8_t *found);
uint64_t pgo_bulk_remove(pgo_table *t, const uint64_t *keys, uint64_t n, uint8_t *ok);

/* occupied slots of a level (count_fill_kernel semantics: non-empty slots,
 * tombstones included) */
uint64_t pgo_count_fill(const pgo_table *t, int level);

/* Multithreaded host port of the same semantics (CAS on the same slot
 * layout, one key per worker step); this is the timed CPU baseline.
 * nthreads <= 0 means all online cores.  Returns insert failures / hits. */
uint64_t pgo_mt_bulk_insert(pgo_table *t, const uint64_t *keys, const uint64_t *vals, uint64_t n, uint8_t *ok, int nthreads);
uint64_t pgo_mt_bulk_query(pgo_table *t, const uint64_t *keys, uint64_t n, uint64_t *vals, uint8_t *found, int nthreads);
uint64_t pgo_mt_bulk_remove(pgo_table *t, const uint64_t *keys, uint64_t n, uint8_t *ok, int nthreads);
int pgo_online_cores(void);

/* slab allocator model: counts of a fixed-size object pool */
typedef struct pgo_slab pgo_slab;
pgo_slab *pgo_slab_create(uint64_t num_allocs);
void pgo_slab_destroy(pgo_slab *s);
uint64_t pgo_slab_capacity(const pgo_slab *s);
uint64_t pgo_slab_free_objects(const pgo_slab *s);
uint64_t pgo_slab_malloc(pgo_slab *s, uint64_t n, uint64_t *offsets);
uint64_t pgo_slab_free(pgo_slab *s, uint64_t n, const uint64_t *offsets);

/* Bucketed two-choice filter with tombstone reuse (tables/bucketed_table.cuh
 * over packed_bucket + grouped_bits_pair slots): poggers_oracle_bucketed.c.
 * tag_bits 16: 4-byte slots (16-bit tag, 16-bit value), tag_bits 8: 2-byte
 * slots.  Levels use PGO_SCHEME_TWO_CHOICE_BUCKETED or PGO_SCHEME_LINEAR_BUCKETED. */
enum {
    PGO_BOP_INSERT = 0,
    PGO_BOP_QUERY = 1,
    PGO_BOP_REMOVE = 2,
    PGO_BOP_INSERT_DELETE = 3,               /* insert_with_delete */
    PGO_BOP_INSERT_IF_NOT_EXISTS = 4,
    PGO_BOP_INSERT_IF_NOT_EXISTS_DELETE = 5
};
typedef struct pgo_bcfg {
    uint32_t tag_bits;
    uint32_t nlevels;
    uint32_t pad0, pad1;
    pgo_level_cfg lv[2];
} pgo_bcfg;
typedef struct pgo_btable pgo_btable;
uint64_t pgo_btag(uint32_t bits, uint64_t key);
pgo_btable *pgo_btable_create(const pgo_bcfg *cfg, uint64_t seed);
void pgo_btable_destroy(pgo_btable *t);
uint64_t pgo_btable_level_bytes(const pgo_btable *t, int level);
uint64_t pgo_btable_level_nbuckets(const pgo_btable *t, int level);
void *pgo_btable_level_data(pgo_btable *t, int level);
/* one operation; *out = value found (query / insert_if_not_exists*), *found = found_val */
int pgo_btable_op(pgo_btable *t, int op, uint64_t key, uint64_t val, uint64_t *out, int *found);
/* sequential bulk form in batch order; returns how many calls returned true */
uint64_t pgo_btable_bulk(pgo_btable *t, int op, const uint64_t *keys, const uint64_t *vals, uint64_t n,
                         uint64_t *out, uint8_t *ok, uint8_t *found);
uint64_t pgo_btable_count_fill(const pgo_btable *t, int level);

/* restatement of the reference's one_size_slab_allocator<E> (poggers_oracle_slabref.c):
 * per-SM pinned slabs, whole-word claims with a per-SM cache, pivot and pool */
typedef struct pgo_rslab pgo_rslab;
enum { PGO_RSLAB_REFUSED = 0, PGO_RSLAB_FREED = 1, PGO_RSLAB_RETURNED = 2, PGO_RSLAB_EMPTIED_PINNED = 3 };
pgo_rslab *pgo_rslab_create(uint64_t num_allocs, int sms, int extra_blocks, uint64_t seed);
void pgo_rslab_destroy(pgo_rslab *a);
uint64_t pgo_rslab_report_fill(const pgo_rslab *a);
uint64_t pgo_rslab_report_max(const pgo_rslab *a);
uint64_t pgo_rslab_short_pins(const pgo_rslab *a);
uint64_t pgo_rslab_lost_words(const pgo_rslab *a);
/* one malloc() call by `group` threads of one warp (1..32) on SM `sm`, served
 * together; out[i] = object offset or ~0; returns the NULL count */
uint64_t pgo_rslab_malloc(pgo_rslab *a, int sm, int group, uint64_t *out);
/* one free(); returns PGO_RSLAB_* */
int pgo_rslab_free(pgo_rslab *a, uint64_t offset);

/* splitmix64 key stream: key i = mix(seed + (i+1) * 0x9E3779B97F4A7C15) */
void pgo_splitmix64_fill(uint64_t seed, uint64_t start, uint64_t n, uint64_t *out);

#ifdef __cplusplus
}
#endif

#endif
