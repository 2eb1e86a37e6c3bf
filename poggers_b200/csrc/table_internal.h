// table_internal.h -- the table object behind the C ABI's opaque pg_table.
#pragma once
#include <stdint.h>
#include "poggers_b200.h"
#include "poggers_b200/level.cuh"
#include <cuda_runtime.h>
#include "on_device.h"

struct pg_table {
    pg_table_config cfg;
    pg::table_desc desc;
    void *mem[2];
    uint64_t bytes[2];
    void *fp;           // fingerprint bytes of level 0 (PG_TABLE_FINGERPRINTS)
    uint64_t fp_bytes;
    int device;
    int num_sms;
    uint32_t block_threads;
    uint32_t blocks_per_sm;
    uint32_t max_blocks;
    uint32_t lanes;  // lanes per key set by pg_table_set_launch; 0 = chosen per operation (pg_table_lanes)
    uint32_t ifmt;  // internal format: public format, split variant when PG_TABLE_SPLIT_BUCKETS
    uint32_t partition;  // region-ordered inserts enabled
    void *part_buf;      // their scratch (keys, values, original index, region counts)
    uint64_t part_bytes;
};

// lanes per key the kernels use for one operation (0 insert, 1 query, 2 remove)
uint32_t pg_table_lanes(const pg_table *t, int op = 1);

namespace pg { struct bulk_args; }
// Region-ordered insert (partition.cu): true when it rewrote `a` to the sorted
// copy; `only` then marks the keys of the caller's batch left for a second pass.
bool pg_partition_insert(pg_table *t, pg::bulk_args &a, const uint32_t *&only, cudaStream_t s);
// Grow that scratch for batches of up to max_keys (stream-ordered); false if it cannot be allocated.
bool pg_partition_reserve(pg_table *t, uint64_t max_keys, cudaStream_t s);
