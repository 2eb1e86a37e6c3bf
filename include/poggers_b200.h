/*
 * poggers_b200.h -- C ABI of the poggers_b200 library (libpoggers_b200.so).
 *
 * B200-native (sm_100a) bulk operations on the POGGERS tables: the
 * Two-Choice Filter (TCF) and the modular uint64 hash tables (double,
 * linear and power-of-two probing over tile-cooperative buckets).
 *
 * Conventions (mirroring the reference where it has one):
 *  - The library owns table memory; the caller owns every key, value and
 *    result buffer.  Buffers passed as d_* are device pointers.
 *  - Every bulk call is asynchronous and ordered on the given stream
 *    (NULL = the legacy default stream).  Calls on the same table must be
 *    phase-separated by stream order: the reference's guarantee that a query
 *    sees an insert holds only across kernel boundaries, and so does ours.
 *  - Tables, batches, servers and allocators live on the device current when
 *    they are created; every later call on one must be made with that device
 *    current, or it returns PG_ERR_INVALID and launches nothing.
 *  - Errors are status codes, never exceptions or device traps.  The
 *    reference throws std::runtime_error on a sizing mismatch
 *    (tables/base_table.cuh:116-131) and returns bool from device ops.
 *  - Counters passed as d_count are ADDED to (like the reference test
 *    harness's atomicAdd on a caller-zeroed counter); zero them first.
 *  - Values are typed by the table format: uint64_t for PG_FMT_KV64,
 *    uint16_t for PG_FMT_TAGVAL16 and PG_FMT_PACKED_TAGVAL16, uint8_t for
 *    PG_FMT_PACKED_TAGVAL8; PG_FMT_TAG16 stores no values and reports
 *    0, like key_container::get_val (representations/key_only.cuh:75-77).
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   pg_table_create   <- static_table::generate_on_device(Sizing*, seed)      tables/base_table.cuh:110-145
 *   pg_table_destroy  <- static_table::free_on_device(Table*)                tables/base_table.cuh:147-164
 *   pg_bulk_insert    <- insert(tile, key, val) launched one tile per key     tables/base_table.cuh:167-187,
 *                        with get_num_blocks / get_block_size                 tables/base_table.cuh:321-329
 *                        (bulk driver shape: tests/src/test_mhm_tcf.cu:319-345)
 *   pg_bulk_query     <- query(tile, key, Val&)                               tables/base_table.cuh:273-290
 *                        (driver: tests/src/test_mhm_tcf.cu:457-521)
 *   pg_bulk_remove    <- remove(tile, key)                                    tables/base_table.cuh:292-308
 *                        (driver: tests/src/delete_tests.cu:336-372)
 *   pg_table_count_fill <- count_fill_kernel / get_fill                       tables/bucketed_table.cuh:37-52,498-548
 *   pg_table_bytes    <- host_bytes_in_use                                    tables/base_table.cuh:331-351
 *   pg_bulk_insert_with_delete <- bucketed_table::insert_with_delete          tables/bucketed_table.cuh:222-240
 *                        (driver: tests/src/delete_tests.cu:274-296)
 *   pg_bulk_insert_if_not_exists[_delete] <- bucketed_table::insert_if_not_exists[_delete]
 *                                                                             tables/bucketed_table.cuh:188-220
 */
#ifndef POGGERS_B200_H
#define POGGERS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ABI-compatible with cudaStream_t, without requiring the CUDA headers. */
typedef struct CUstream_st *pg_stream_t;

typedef enum pg_status {
    PG_OK = 0,
    PG_ERR_INVALID = 1,     /* bad argument or configuration */
    PG_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    PG_ERR_NOMEM = 3,       /* device allocation failed */
    PG_ERR_UNSUPPORTED = 4, /* valid but not compiled in (bucket size / tile combination) */
    PG_ERR_FULL = 5,        /* capacity exhausted */
    PG_ERR_TIMEOUT = 6,     /* a bounded device wait gave up */
    PG_ERR_TOO_LARGE = 7    /* more tables or requests than the fixed scratch of pg_batch_run_static holds */
} pg_status;

/* slot formats (reference representations) */
enum {
    PG_FMT_KV64 = 0,     /* key_val_pair<uint64_t,uint64_t>: the modular hash tables */
    PG_FMT_TAGVAL16 = 1, /* dynamic_container<key_val_pair,uint16_t>: the TCF (16-bit tag + 16-bit val) */
    PG_FMT_TAG16 = 2,    /* dynamic_container<key_container,uint16_t>: tag-only TCF */
    /* the bucketed filter with tombstone reuse: bucketed_internal_dynamic_container
     * of grouped_bits_pair slots, one CAS-able word per slot (tag low, value high);
     * used with the *_BUCKETED schemes on every level (tests/src/delete_tests.cu:138-179) */
    PG_FMT_PACKED_TAGVAL16 = 3, /* grouped_bits_pair<16,16>: 4-byte slots (del_TCF) */
    PG_FMT_PACKED_TAGVAL8 = 4   /* grouped_bits_pair<8,8>: 2-byte slots (del_TCF_small) */
};

/* insert schemes */
enum {
    PG_SCHEME_BUCKET = 0,     /* insert_schemes/bucket_insert.cuh */
    PG_SCHEME_TWO_CHOICE = 1, /* insert_schemes/power_of_n_shortcut.cuh (max_probes <= 4) */
    PG_SCHEME_TWO_CHOICE_BUCKETED = 2, /* insert_schemes/power_of_n_shortcut_buckets.cuh (max_probes <= 4,
                                          bucket 8/16/32; packed formats only) */
    PG_SCHEME_LINEAR_BUCKETED = 3      /* insert_schemes/linear_insert_buckets.cuh (packed formats only;
                                          bucket 8/16/32 as primary, 8/16 as backing) */
};

/* probing schemes */
enum {
    PG_PROBE_DOUBLE = 0,  /* probing_schemes/double_hashing.cuh */
    PG_PROBE_LINEAR = 1,  /* probing_schemes/linear_probing.cuh */
    PG_PROBE_P2 = 2,      /* probing_schemes/power_of_two.cuh (max_probes == 2) */
    PG_PROBE_XOR_P2 = 3   /* probing_schemes/xor_power_of_two.cuh (max_probes == 2) */
};

typedef struct pg_level_config {
    uint64_t nslots;      /* requested slots; buckets = ceil(nslots / bucket_size) */
    uint32_t bucket_size; /* level 0: 4, 8, 16 or 32; level 1: 1..64 */
    uint32_t max_probes;
    uint32_t scheme;      /* PG_SCHEME_* */
    uint32_t probe;       /* PG_PROBE_* */
} pg_level_config;

/* table flags */
enum {
    /* Keep each bucket's keys contiguous, then its values ([B keys | B vals]),
     * instead of the reference's {key, val} slots.  Same results, and dumps
     * and images still use the reference's layout; a probe reads the keys
     * without the values (for the TCF's 16-bit tags, one 32-byte sector per
     * bucket). */
    PG_TABLE_SPLIT_BUCKETS = 1u,
    /* uint64 tables (PG_FMT_KV64, bucket_insert primary, reference layout):
     * keep one fingerprint byte per slot in a separate array (1/16 of the
     * slot bytes) that the kernels hold in L2, so probes touch DRAM only for
     * slots whose fingerprint matches.  Same results. */
    PG_TABLE_FINGERPRINTS = 2u
};

typedef struct pg_table_config {
    uint32_t format;   /* PG_FMT_* */
    uint32_t tile;     /* lanes per key (the reference's Partition_Size): 1,2,4,8,16; <= level-0 bucket size */
    uint32_t nlevels;  /* 1, or 2 = primary + backing (static_table's recursive table) */
    uint32_t flags;    /* PG_TABLE_* bits, 0 = the reference's slot layout */
    pg_level_config levels[2];
} pg_table_config;

typedef struct pg_level_info {
    uint64_t nbuckets;
    uint64_t nslots;       /* nbuckets * bucket_size */
    uint64_t bytes;        /* device bytes of the bucket array */
    uint64_t seed;         /* level seed (level 0: the table seed, level 1: seed*seed) */
    const void *d_buckets; /* device address of the bucket array */
} pg_level_info;

typedef struct pg_table pg_table;

/* Library version string, e.g. "poggers_b200 0.1 sm_100a". */
const char *pg_version(void);
const char *pg_status_string(pg_status s);

/* Create a table on the current device; slot arrays are zeroed.  Level l is
 * hashed with seed^(2^l) exactly like static_table::generate_on_device. */
pg_status pg_table_create(const pg_table_config *cfg, uint64_t seed, pg_table **out);
pg_status pg_table_destroy(pg_table *t);
/* Zero every slot (stream-ordered). */
pg_status pg_table_clear(pg_table *t, pg_stream_t stream);
pg_status pg_table_level_info(const pg_table *t, uint32_t level, pg_level_info *out);
/* Device bytes owned by the table (host_bytes_in_use). */
uint64_t pg_table_bytes(const pg_table *t);

/* Launch shape of the bulk kernels: threads per block (<= 256, a multiple of
 * the lanes per key; 0 = 256), blocks per SM (0 = 32), a cap on blocks (0 =
 * none) and the lanes that serve one key (1, 2, 4, 8 or 16, at most the
 * level-0 bucket size; packed formats run 1 or 4 lanes).  Lanes 0, the
 * default of a new table, chooses them per operation by measurement: one
 * lane per key, except two for queries and removes of uint64 tables without
 * fingerprints, and four (the reference's tile) for inserts into a
 * two-choice level of fewer than 2^18 slots, where one lane per key puts the
 * whole batch in flight at once and unbalances the two choices.  The lanes per key never change a
 * result: filled slots always form a prefix of each bucket, so the
 * reference's tile-wide stripes decide exactly what a whole-bucket scan
 * decides.  block_threads == lanes with max_blocks == 1 runs the batch
 * strictly in order on one group (the reference's serial layout). */
pg_status pg_table_set_launch(pg_table *t, uint32_t block_threads, uint32_t blocks_per_sm, uint32_t max_blocks,
                              uint32_t lanes_per_key);

/* ---------------------------------------------------------------------------
 * One logical table partitioned over several GPUs (no counterpart in the
 * reference, whose tables live on one GPU).  Key k belongs to shard
 * pg_host_shard_of(k, route_seed, nshards) = high bits of
 * MurmurHash64A(k, route_seed) * nshards; each GPU holds its shard as an
 * ordinary table.  A bulk call routes its batch (pg_route_by_shard), the
 * caller exchanges the per-shard runs with an all-to-all (NCCL), each GPU
 * runs the bulk operation on what it received, the results travel back by
 * the reverse all-to-all and pg_scatter_by_perm puts them in batch order
 * (poggers_b200/sharded.py does all of this over torch.distributed). */
uint32_t pg_host_shard_of(uint64_t key, uint64_t route_seed, uint32_t nshards);
/* Counting sort of n < 2^32 keys (and values of val_bytes 0, 1, 2 or 8) by
 * shard: d_keys_out / d_vals_out hold the shards' runs in shard order,
 * d_perm_out[i] = the batch position of output i, d_counts[0..nshards) = run
 * lengths; d_counts must hold 2 * nshards entries (the second half is
 * scratch).  nshards <= 1024.  Stream-ordered. */
pg_status pg_route_by_shard(const uint64_t *d_keys, const void *d_vals, uint32_t val_bytes, uint64_t n,
                            uint32_t nshards, uint64_t route_seed, uint64_t *d_keys_out, void *d_vals_out,
                            uint32_t *d_perm_out, uint64_t *d_counts, pg_stream_t stream);
/* d_dst[d_perm[i]] = d_src[i] for elements of 1, 2 or 8 bytes. */
pg_status pg_scatter_by_perm(const void *d_src, const uint32_t *d_perm, uint64_t n, uint32_t elem_bytes, void *d_dst,
                             pg_stream_t stream);

/* Region-ordered inserts (on by default; enable = 0 turns them off).  A
 * batch of at least 2^20 keys into a uint64 bucket table of at least 64 MB
 * is first sorted by the table region (32 MB) of each key's first bucket,
 * into one run per region, then inserted in that order, so each bucket line
 * is fetched from HBM once for all its keys instead of once per key.  A run
 * holds the keys expected in its region plus a margin; the keys a run cannot
 * hold (a batch far from uniform over the table) are inserted afterwards in
 * batch order.  The sort costs about 20 bytes of device scratch per key,
 * kept by the table (counted in pg_table_bytes) until pg_table_destroy.  The
 * first such insert (or one larger than any before) grows it with a
 * stream-ordered allocation on the insert's stream (cudaMallocAsync: no
 * device-wide synchronization); pg_table_reserve_insert_scratch grows it
 * ahead of time, so that no insert allocates.
 * Concurrent inserts have no defined order in the reference either: which
 * keys fail when a table overflows may differ, every placed key is
 * placed by the same rule.  The scratch is the table's: two region-ordered
 * inserts into one table must be ordered on one stream. */
pg_status pg_table_set_partitioned_insert(pg_table *t, int enable);
/* Whether a fingerprinted table's fingerprint array is treated as L2-resident
 * (default: when it is at most 80 MB).  Resident, its loads are marked
 * evict-last and a query reads two buckets' fingerprints per step; not
 * resident, loads are plain and a query reads one bucket per step.  Results
 * are the same either way.  Batches take the setting when they are created.
 * PG_ERR_INVALID for a table without fingerprints.  No counterpart in the
 * reference. */
pg_status pg_table_set_fingerprint_residency(pg_table *t, int resident);
/* Grow the region sort's scratch for insert batches of up to max_batch_keys
 * keys (ordered on `stream`); PG_ERR_NOMEM if it cannot be allocated.  No
 * counterpart in the reference. */
pg_status pg_table_reserve_insert_scratch(pg_table *t, uint64_t max_batch_keys, pg_stream_t stream);

/* Bulk insert of n keys (and values; d_vals may be NULL = all 0).
 * d_ok[i] (optional) = 1 if key i was placed; d_fail_count (optional) += failures.
 * Replaces the reference's per-tile insert loop over a batch
 * (tables/base_table.cuh:174-214, driven one key per tile by its tests). */
pg_status pg_bulk_insert(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n,
                         uint8_t *d_ok, uint64_t *d_fail_count, pg_stream_t stream);

/* Bulk query: d_vals_out[i] (optional) = value found (0 if absent);
 * d_found[i] (optional) = 1 if present; d_hit_count (optional) += hits. */
pg_status pg_bulk_query(pg_table *t, const uint64_t *d_keys, uint64_t n, void *d_vals_out,
                        uint8_t *d_found, uint64_t *d_hit_count, pg_stream_t stream);

/* Bulk remove (tombstones): d_ok[i] (optional) = 1 if a matching slot was
 * removed; d_hit_count (optional) += removals. */
pg_status pg_bulk_remove(pg_table *t, const uint64_t *d_keys, uint64_t n, uint8_t *d_ok,
                         uint64_t *d_hit_count, pg_stream_t stream);

/* Bucketed filter (packed formats) only; other formats return PG_ERR_UNSUPPORTED,
 * as the reference's static_table schemes have no such methods.
 *
 * insert_with_delete: like pg_bulk_insert, but a deleted slot may be reused
 * (packed_bucket.cuh:116-180).  d_ok / d_fail_count as for pg_bulk_insert. */
pg_status pg_bulk_insert_with_delete(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n,
                                     uint8_t *d_ok, uint64_t *d_fail_count, pg_stream_t stream);
/* insert_if_not_exists: a key already present is reported (d_found[i] = 1,
 * d_vals_out[i] = its value) and not inserted again; otherwise it is inserted.
 * d_ok[i] = 1 when found or inserted; d_fail_count += keys neither found nor
 * inserted.  The _delete form removes a key it finds instead (the
 * reference's find-and-delete), reusing deleted slots when it inserts. */
pg_status pg_bulk_insert_if_not_exists(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n,
                                       void *d_vals_out, uint8_t *d_found, uint8_t *d_ok, uint64_t *d_fail_count,
                                       pg_stream_t stream);
pg_status pg_bulk_insert_if_not_exists_delete(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n,
                                              void *d_vals_out, uint8_t *d_found, uint8_t *d_ok,
                                              uint64_t *d_fail_count, pg_stream_t stream);

/* d_out[0] += occupied (non-empty) slots of `level`, d_out[1] += tombstones.
 * The bucketed filter's get_fill (live slots) is d_out[0] - d_out[1]. */
pg_status pg_table_count_fill(pg_table *t, uint32_t level, uint64_t *d_out, pg_stream_t stream);

/* Copy a level to / from host memory in the REFERENCE's slot layout
 * (array of {key, val} structs, buckets of bucket_size consecutive slots),
 * so dumps compare byte-for-byte with the reference's device table and can
 * be reloaded.  `bytes` must equal nslots * slot size (16, 4 or 2 bytes).
 * Synchronous. */
pg_status pg_table_dump_level(const pg_table *t, uint32_t level, void *host_dst, uint64_t bytes);
pg_status pg_table_load_level(pg_table *t, uint32_t level, const void *host_src, uint64_t bytes);

/* Checkpoint image of a whole table, for save / restore of resident tables
 * (no counterpart in the reference, which has no on-disk form).  Layout,
 * little-endian: a 128-byte header (magic "PGB2TBL1", version 1, header
 * size, the pg_table_config, the seed, each level's byte count, an FNV-1a
 * 64 checksum of the payload), then every level in the reference's slot
 * layout (pg_table_dump_level).  Synchronous. */
#define PG_IMAGE_HEADER_BYTES 128
uint64_t pg_table_image_bytes(const pg_table *t);
pg_status pg_table_save_image(const pg_table *t, void *host_dst, uint64_t bytes);
/* Create a table on the current device from an image.  A short, corrupt or
 * foreign image returns PG_ERR_INVALID before anything is allocated. */
pg_status pg_table_load_image(const void *host_src, uint64_t bytes, pg_table **out);

/* ---------------------------------------------------------------------------
 * Multi-table batches: many requests over many tables in one persistent launch.
 *
 * No counterpart in the reference, which launches one kernel per batch per
 * table (tests/src/test_mhm_tcf.cu:603-685); each request here is what one
 * such launch would do, and its results equal that launch's.  Requests in one
 * run execute concurrently, so -- as with separate launches -- requests that
 * conflict on one table (an insert or remove with anything else on that
 * table) belong in separate runs (stream-ordered).
 * --------------------------------------------------------------------------- */
/* PG_OP_INSERT_WITH_DELETE: bucketed_table::insert_with_delete, for tables of
 * the packed formats only (requests of it on other tables are skipped). */
enum { PG_OP_INSERT = 0, PG_OP_QUERY = 1, PG_OP_REMOVE = 2, PG_OP_INSERT_WITH_DELETE = 3 };

typedef struct pg_op_desc {
    uint32_t table;  /* index into the batch's table list */
    uint32_t op;     /* PG_OP_* */
    uint64_t offset; /* first key (and value / result) index of the request */
    uint64_t count;  /* keys in the request */
} pg_op_desc;

typedef struct pg_batch pg_batch;

/* Register tables for batched runs.  All must share format, layout flags,
 * level-0 bucket size and scheme, and whether they have a backing level.
 * max_ops bounds the requests of one run (scratch is sized for it). */
pg_status pg_batch_create(pg_table *const *tables, uint32_t ntables, uint32_t max_ops, pg_batch **out);
pg_status pg_batch_destroy(pg_batch *b);
pg_status pg_batch_set_launch(pg_batch *b, uint32_t block_threads, uint32_t blocks_per_sm, uint32_t lanes_per_key);
/* Clear every table of the batch (what pg_table_clear does to each: all levels
 * and fingerprint arrays zeroed) with one kernel launch, so a captured graph of
 * a whole batch step holds one clear instead of a memset per table and level.
 * No counterpart in the reference. */
pg_status pg_batch_clear(pg_batch *b, pg_stream_t stream);
/* Run d_ops[0 .. *d_nops) (both device memory, so one captured CUDA graph can be
 * replayed with new requests).  Keys, values and per-key flags are indexed by
 * the requests' offsets; d_op_counts[j] (optional) += hits of query / remove
 * request j, or failures of insert request j. */
pg_status pg_batch_run(pg_batch *b, const pg_op_desc *d_ops, const uint32_t *d_nops, const uint64_t *d_keys,
                       const void *d_vals_in, void *d_vals_out, uint8_t *d_flags, uint64_t *d_op_counts,
                       pg_stream_t stream);

/* Allocation-free variant of pg_batch_run, for callers that cannot call
 * cudaMalloc (code running inside another allocator, a plugin whose host
 * forbids device allocations, or a process whose device memory is fully
 * budgeted).  No counterpart in the reference.  It takes the tables directly
 * (no pg_batch object) and keeps everything it needs besides the caller's
 * inputs and outputs -- the tables' device descriptors, the per-request chunk
 * offsets and the work counter -- in one fixed array compiled into the
 * library, at most PG_STATIC_MAX_TABLES tables and PG_STATIC_MAX_OPS requests
 * per call (larger calls return PG_ERR_TOO_LARGE).  That array (about 106 KB)
 * exists once on every GPU that loads the library, until the process exits.
 *  - The first call on a device looks up the array's device address and keeps
 *    it for the process's life, so do not use the call across a
 *    cudaDeviceReset().
 *  - The current device must be the tables' device (else PG_ERR_INVALID,
 *    before anything is launched).
 *  - Every call shares the array and leaves its contents behind (the work
 *    counter is reset by each call), so calls whose work overlaps on the GPU
 *    (different streams, or different host threads) race: order them.
 *  - It allocates no device memory and calls no allocating library routine;
 *    results equal pg_batch_run's for the same tables and requests. */
#define PG_STATIC_MAX_TABLES 256
#define PG_STATIC_MAX_OPS 8192
pg_status pg_batch_run_static(pg_table *const *tables, uint32_t ntables, const pg_op_desc *d_ops,
                              const uint32_t *d_nops, uint32_t max_ops, const uint64_t *d_keys,
                              const void *d_vals_in, void *d_vals_out, uint8_t *d_flags, uint64_t *d_op_counts,
                              pg_stream_t stream);

/* ---------------------------------------------------------------------------
 * Continuous-batching server over resident tables (no counterpart in the
 * reference).  Requests from host memory are packed by a worker thread into
 * waves of pg_batch_run calls; up to two waves are on the GPU at once, and
 * requests that arrive meanwhile join the next wave.  Per table, requests
 * complete in submission order and results equal running them one at a
 * time in that order.  A request's host buffers must stay valid until it
 * completes.
 * --------------------------------------------------------------------------- */
typedef struct pg_server pg_server;

typedef struct pg_server_config {
    uint64_t hbm_budget_bytes;  /* tables are admitted while their bytes fit */
    uint64_t max_wave_keys;     /* keys staged per wave (also the largest request) */
    uint32_t max_wave_requests; /* requests per wave */
    uint32_t reserved;
} pg_server_config;

pg_status pg_server_create(const pg_server_config *cfg, pg_server **out);
pg_status pg_server_destroy(pg_server *s);
/* Create a resident table; PG_ERR_FULL when it would exceed the HBM budget. */
pg_status pg_server_add_table(pg_server *s, const pg_table_config *cfg, uint64_t seed, uint32_t *table_id);
/* Release a table and its share of the budget (none of its requests may be pending). */
pg_status pg_server_drop_table(pg_server *s, uint32_t table_id);
pg_table *pg_server_table(pg_server *s, uint32_t table_id);
uint64_t pg_server_bytes_in_use(pg_server *s);
/* Queue one request; values typed as for pg_bulk_*.  h_vals_out / h_flags optional. */
pg_status pg_server_submit(pg_server *s, uint32_t table_id, uint32_t op, const uint64_t *h_keys, const void *h_vals,
                           uint64_t n, void *h_vals_out, uint8_t *h_flags, uint64_t *request_id);
/* Collect a finished request: PG_OK (count = hits or failures, latency in
 * seconds from submit to completion), or PG_ERR_TIMEOUT if it is still
 * running and wait == 0.  A request is collected once; an id that was never
 * issued or was already collected returns PG_ERR_INVALID (it does not wait). */
pg_status pg_server_poll(pg_server *s, uint64_t request_id, int wait, uint64_t *count, double *latency_s);
/* Slab size-class sets served by the loop (as pg_slab_set_create; their pools
 * count against the HBM budget, PG_ERR_FULL when they would not fit).
 * PG_OP_MALLOC requests take n object sizes (uint32_t) and return n object
 * pointers (NULL where none was left; count = NULLs); PG_OP_FREE requests take
 * n pointers (count = refused frees).  Requests on one set complete in
 * submission order, and a wave never mixes mallocs and frees of one set. */
enum { PG_OP_MALLOC = 4, PG_OP_FREE = 5 };
pg_status pg_server_add_slab_set(pg_server *s, uint32_t nclasses, const uint64_t *class_bytes,
                                 const uint64_t *num_allocs, uint32_t *set_id);
pg_status pg_server_submit_slab(pg_server *s, uint32_t set_id, uint32_t op, const void *h_in, uint64_t n,
                                uint64_t *h_ptrs_out, uint64_t *request_id);
pg_status pg_server_stats(pg_server *s, uint64_t *waves, uint64_t *keys);
/* Where the server's worker thread spent its time since creation (seconds):
 * planning waves (with the lock held), copying request inputs into pinned
 * staging, issuing the wave's copies and runs, copying results out to the
 * clients' buffers, and waiting -- with waves in flight and no free slot or
 * nothing pending (busy), or with nothing in flight (idle). */
typedef struct pg_server_timing_t {
    uint64_t waves, requests, keys;
    double plan_s, copy_in_s, issue_s, copy_out_s, wait_busy_s, wait_idle_s;
} pg_server_timing_t;
pg_status pg_server_timing(pg_server *s, pg_server_timing_t *out);

/* ---------------------------------------------------------------------------
 * Slab allocator: fixed-size objects from slabs of 4096.
 *
 * Replaces one_size_slab_allocator<N> (allocators/slab_one_size.cuh:58-659):
 *   pg_slab_create        <- generate_on_device(num_allocs, size)     slab_one_size.cuh:84-140
 *   pg_slab_destroy       <- free_on_device                            slab_one_size.cuh:142-180
 *   pg_slab_bulk_malloc   <- malloc() one thread per allocation        slab_one_size.cuh:186-288
 *                            (driver: tests/src/slab_one_size_tests.cu:72-104)
 *   pg_slab_bulk_free     <- free(void*)                               slab_one_size.cuh:428-463
 *   pg_slab_report        <- report_fill / report_max                  slab_one_size.cuh:628-654
 * Capacity is ceil(num_allocs / 4096) * 4096 objects.  A malloc that finds no
 * object after 25 bounded attempts returns NULL, like the reference.
 * --------------------------------------------------------------------------- */
typedef struct pg_slab pg_slab;
typedef struct pg_slab_set pg_slab_set;

#define PG_SLAB_MAX_CLASSES 16

typedef struct pg_slab_info_t {
    void *pool;               /* device address of object 0 */
    uint64_t pool_bytes;
    uint64_t object_bytes;
    uint64_t capacity;        /* objects */
    uint64_t nslabs;
    uint64_t *d_stats;        /* device: [0] double frees, [1] frees of foreign / misaligned pointers */
} pg_slab_info_t;

pg_status pg_slab_create(uint64_t num_allocs, uint64_t object_bytes, pg_slab **out);
pg_status pg_slab_destroy(pg_slab *a);
/* Mark every object free again (stream-ordered). */
pg_status pg_slab_reset(pg_slab *a, pg_stream_t stream);
pg_status pg_slab_info(const pg_slab *a, pg_slab_info_t *out);
/* d_ptrs[i] = a distinct object or NULL; d_fail_count (optional) += NULLs. */
pg_status pg_slab_bulk_malloc(pg_slab *a, uint64_t n, void **d_ptrs, uint64_t *d_fail_count, pg_stream_t stream);
/* Free d_ptrs[0..n) (NULL entries are skipped); d_bad_count (optional) +=
 * double frees and pointers that are not objects of this pool. */
pg_status pg_slab_bulk_free(pg_slab *a, void *const *d_ptrs, uint64_t n, uint64_t *d_bad_count, pg_stream_t stream);
/* d_out[0] += free objects, d_out[1] += fully free slabs. */
pg_status pg_slab_count_free(pg_slab *a, uint64_t *d_out, pg_stream_t stream);
/* Synchronous report: free slabs (report_fill), slabs (report_max), free objects, double frees. */
pg_status pg_slab_report(pg_slab *a, uint64_t *free_slabs, uint64_t *max_slabs, uint64_t *free_objects,
                         uint64_t *double_frees);

/* The device-side descriptor of the pool, for device callers compiled against
 * include/poggers_b200/slab.cuh (the template API's one_size_slab_allocator
 * copies it into its device struct): `bytes` must equal sizeof(pg::slab_desc).
 * Replaces the device struct that one_size_slab_allocator::generate_on_device
 * builds (allocators/slab_one_size.cuh:84-141). */
pg_status pg_slab_desc(const pg_slab *a, void *out_desc, uint64_t bytes);

/* Size classes: one pool per class (class_bytes strictly increasing, at most
 * PG_SLAB_MAX_CLASSES).  A request of s bytes is served by the smallest class
 * with class_bytes >= s; larger requests get NULL. */
pg_status pg_slab_set_create(uint32_t nclasses, const uint64_t *class_bytes, const uint64_t *num_allocs,
                             pg_slab_set **out);
pg_status pg_slab_set_destroy(pg_slab_set *s);
pg_slab *pg_slab_set_class(pg_slab_set *s, uint32_t c);
pg_status pg_slab_set_bulk_malloc(pg_slab_set *s, const uint32_t *d_sizes, uint64_t n, void **d_ptrs,
                                  uint64_t *d_fail_count, pg_stream_t stream);
pg_status pg_slab_set_bulk_free(pg_slab_set *s, void *const *d_ptrs, uint64_t n, uint64_t *d_bad_count,
                                pg_stream_t stream);

/* ---------------------------------------------------------------------------
 * Pinned slab pool: the reference's own slab policy, whose NULL returns,
 * report_fill and free counters equal the reference's on the same calls.
 * Every SM pins a primary slab and extra_blocks backups when the pool is
 * created; a malloc claims a whole 64-object word of the primary and keeps
 * the objects it does not use in its SM's cache; when the primary has no whole
 * word left a backup takes its place and the pool refills the backup's place.
 * So a malloc can return NULL while other SMs' slabs still hold free objects,
 * and report_fill counts only the slabs in the pool.  (pg_slab_create's pool
 * returns NULL only when the whole pool is full.)  The template API's
 * one_size_slab_allocator<extra_blocks> is built on this pool.
 *   pg_pslab_create       <- one_size_slab_allocator<E>::generate_on_device  slab_one_size.cuh:84-141
 *                            (pins: smid_pinned_container::generate_on_device offset_slab.cuh:1838-1873)
 *   pg_pslab_bulk_malloc  <- malloc() one thread per allocation         slab_one_size.cuh:186-288
 *   pg_pslab_bulk_free    <- free / free_count_misses                   slab_one_size.cuh:428-506
 *   pg_pslab_report       <- report_fill / report_max                   slab_one_size.cuh:628-654
 * --------------------------------------------------------------------------- */
typedef struct pg_pslab pg_pslab;
/* Pool of ceil(num_allocs / 4096) slabs; extra_blocks backups per SM (< 63).
 * Synchronous; SM ids are those below the device's %nsmid. */
pg_status pg_pslab_create(uint64_t num_allocs, uint64_t object_bytes, uint32_t extra_blocks, pg_pslab **out);
pg_status pg_pslab_destroy(pg_pslab *a);
/* Device descriptor for device callers of include/poggers_b200/slab_pinned.cuh;
 * `bytes` must equal sizeof(pg::pslab_desc). */
pg_status pg_pslab_desc(const pg_pslab *a, void *out_desc, uint64_t bytes);
/* Synchronous report: slabs in the pool (report_fill), slabs (report_max),
 * SM ids with pins, double frees seen. */
pg_status pg_pslab_report(const pg_pslab *a, uint64_t *pool_slabs, uint64_t *max_slabs, uint64_t *sm_ids,
                          uint64_t *double_frees);
/* d_ptrs[i] = an object or NULL, one malloc() per thread; d_fail_count (optional) += NULLs. */
pg_status pg_pslab_bulk_malloc(pg_pslab *a, uint64_t n, void **d_ptrs, uint64_t *d_fail_count, pg_stream_t stream);
/* The serial launch shape: one warp makes `rounds` malloc() calls of `group`
 * lanes (1..32) each, in order; d_ptrs[k * group + lane]. */
pg_status pg_pslab_serial_malloc(pg_pslab *a, uint32_t rounds, uint32_t group, void **d_ptrs, uint64_t *d_fail_count,
                                 pg_stream_t stream);
/* Free d_ptrs[0..n) (NULL entries skipped), one thread per pointer, or in
 * order by one thread when `serial`; d_counts[0..3] += frees refused (double
 * or foreign), frees done, slabs returned to the pool (free_count_misses'
 * misses[0]), slabs emptied while pinned (misses[1]). */
pg_status pg_pslab_bulk_free(pg_pslab *a, void *const *d_ptrs, uint64_t n, uint64_t *d_counts, int serial,
                             pg_stream_t stream);

/* ---------------------------------------------------------------------------
 * Diagnostics (no counterpart in the reference): the GPU's random-access
 * ceilings, which bound the filters' kernels (one or two 32-byte sectors at
 * random addresses per key, and an atomic claim on a sector just read).
 * pg_diag_random_access makes about `accesses` accesses of one kind at
 * hashed random offsets inside d_buf (64-byte aligned, >= 64 bytes), several
 * in flight per thread, on blocks_per_sm (1-8, 0 = 8) blocks of 256 threads
 * per SM; *accesses_done receives the exact count (rounded up to whole
 * per-thread batches).  READ32: one 32-byte sector; READ64: two adjacent
 * sectors; READ32_CAS: one sector, then a CAS on its first 4-byte word with
 * the value read; RED32: an atomic add (no return) on a random 4-byte word;
 * READ32_CAS_NEXT: within a random 64-byte span, READ32_CAS on its first
 * sector and a 2-byte store into its second (a split filter bucket's insert:
 * claim a tag, then write its value).
 * CAS and RED modes modify d_buf.  d_sink (8 bytes) only keeps the loads.
 * --------------------------------------------------------------------------- */
#define PG_DIAG_READ32 0
#define PG_DIAG_READ64 1
#define PG_DIAG_READ32_CAS 2
#define PG_DIAG_RED32 3
#define PG_DIAG_READ32_CAS_NEXT 4
pg_status pg_diag_random_access(void *d_buf, uint64_t bytes, uint32_t mode, uint64_t accesses, uint64_t seed,
                                uint32_t blocks_per_sm, uint64_t *accesses_done, uint64_t *d_sink,
                                pg_stream_t stream);

/* Host-side helpers used by tests (no GPU needed). */
uint64_t pg_host_murmur64a(uint64_t key, uint64_t seed);
uint64_t pg_host_fastmod(uint64_t n, uint64_t d);
/* Bucket ids (after % nbuckets) a table level probes for `key`; returns count. */
uint32_t pg_host_probe_buckets(const pg_table_config *cfg, uint32_t level, uint64_t seed, uint64_t key,
                               uint64_t *out, uint32_t cap);

#ifdef __cplusplus
}
#endif

#endif /* POGGERS_B200_H */
