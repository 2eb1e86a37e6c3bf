// table.cu -- C ABI: table lifetime, bulk-op launchers, fill counts, dumps.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime.h>
#include <vector>

#include "poggers_b200.h"
#include "bulk_kernels.cuh"
#include "bulk_packed.cuh"

using namespace pg;

#include "table_internal.h"

namespace {

// largest fingerprint array kept in L2 with evict-last loads (L2 is 126 MB; the
// slot lines of the buckets in use need the rest)
constexpr uint64_t kFpResidentBytes = 80ull << 20;

bool packed(uint32_t fmt) { return fmt == PG_FMT_PACKED_TAGVAL16 || fmt == PG_FMT_PACKED_TAGVAL8; }
uint32_t key_bytes(uint32_t fmt)
{
    return fmt == PG_FMT_KV64 ? 8u : (fmt == PG_FMT_PACKED_TAGVAL8 ? 1u : 2u);
}
uint32_t val_bytes(uint32_t fmt)
{
    switch (fmt) {
    case PG_FMT_KV64: return 8u;
    case PG_FMT_TAGVAL16:
    case PG_FMT_PACKED_TAGVAL16: return 2u;
    case PG_FMT_PACKED_TAGVAL8: return 1u;
    default: return 0u;
    }
}

bool split_layout(const pg_table_config *c)
{
    return (c->flags & PG_TABLE_SPLIT_BUCKETS) && c->format != PG_FMT_TAG16;
}

bool fingerprinted(const pg_table_config *c)
{
    return (c->flags & PG_TABLE_FINGERPRINTS) != 0;
}

uint32_t internal_format(const pg_table_config *c)
{
    if (c->format == PG_FMT_PACKED_TAGVAL16) return FMT_PACKED16;
    if (c->format == PG_FMT_PACKED_TAGVAL8) return FMT_PACKED8;
    if (fingerprinted(c)) return FMT_KV64_FP;
    if (!split_layout(c)) return c->format;
    return c->format == PG_FMT_KV64 ? (uint32_t)FMT_KV64_SPLIT : (uint32_t)FMT_TAGVAL16_SPLIT;
}

pg_status validate(const pg_table_config *c)
{
    if (!c || (c->flags & ~(uint32_t)(PG_TABLE_SPLIT_BUCKETS | PG_TABLE_FINGERPRINTS)) != 0) return PG_ERR_INVALID;
    if (c->flags & PG_TABLE_FINGERPRINTS) {
        // a fingerprint byte per uint64 slot, on a bucket_insert primary with the reference layout
        if (c->format != PG_FMT_KV64 || (c->flags & PG_TABLE_SPLIT_BUCKETS) || c->nlevels < 1 ||
            c->levels[0].scheme != PG_SCHEME_BUCKET)
            return PG_ERR_UNSUPPORTED;
    }
    if (c->format > PG_FMT_PACKED_TAGVAL8) return PG_ERR_INVALID;
    if (c->nlevels < 1 || c->nlevels > 2) return PG_ERR_INVALID;
    if (!(c->tile == 1 || c->tile == 2 || c->tile == 4 || c->tile == 8 || c->tile == 16)) return PG_ERR_INVALID;
    if (packed(c->format)) {
        // the bucketed filter: packed slots with the bucketed schemes on every level
        if (c->flags) return PG_ERR_UNSUPPORTED;
        for (uint32_t l = 0; l < c->nlevels; l++) {
            const pg_level_config &L = c->levels[l];
            if (L.nslots == 0 || L.bucket_size == 0 || L.max_probes == 0 || L.probe > PG_PROBE_XOR_P2)
                return PG_ERR_INVALID;
            if (L.scheme != PG_SCHEME_TWO_CHOICE_BUCKETED && L.scheme != PG_SCHEME_LINEAR_BUCKETED)
                return PG_ERR_INVALID;
            if ((L.probe == PG_PROBE_P2 || L.probe == PG_PROBE_XOR_P2) && L.max_probes != 2) return PG_ERR_INVALID;
            if (L.scheme == PG_SCHEME_TWO_CHOICE_BUCKETED && L.max_probes > (uint32_t)kTwoChoiceMaxProbes)
                return PG_ERR_UNSUPPORTED;
            if (L.nslots / L.bucket_size > (1ULL << 40)) return PG_ERR_INVALID;
        }
        const uint32_t b0 = c->levels[0].bucket_size;
        if (!(b0 == 8 || b0 == 16 || b0 == 32)) return PG_ERR_UNSUPPORTED;
        if (c->nlevels > 1 && !(c->levels[1].bucket_size == 8 || c->levels[1].bucket_size == 16))
            return PG_ERR_UNSUPPORTED;
        if (c->tile > b0) return PG_ERR_UNSUPPORTED;
        return PG_OK;
    }
    for (uint32_t l = 0; l < c->nlevels; l++) {
        const pg_level_config &L = c->levels[l];
        if (L.nslots == 0 || L.bucket_size == 0 || L.max_probes == 0) return PG_ERR_INVALID;
        if (L.scheme > PG_SCHEME_TWO_CHOICE || L.probe > PG_PROBE_XOR_P2) return PG_ERR_INVALID;
        if ((L.probe == PG_PROBE_P2 || L.probe == PG_PROBE_XOR_P2) && L.max_probes != 2) return PG_ERR_INVALID;
        if (L.scheme == PG_SCHEME_TWO_CHOICE && L.max_probes > (uint32_t)kTwoChoiceMaxProbes) return PG_ERR_UNSUPPORTED;
        if (L.bucket_size > 64) return PG_ERR_UNSUPPORTED;
        if (L.nslots / L.bucket_size > (1ULL << 40)) return PG_ERR_INVALID;
    }
    const uint32_t b0 = c->levels[0].bucket_size;
    if (!(b0 == 4 || b0 == 8 || b0 == 16 || b0 == 32)) return PG_ERR_UNSUPPORTED;
    if (c->tile > b0) return PG_ERR_UNSUPPORTED;
    return PG_OK;
}

pg_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return PG_OK;
    if (e == cudaErrorMemoryAllocation) return PG_ERR_NOMEM;
    if (e == cudaErrorInvalidConfiguration) return PG_ERR_UNSUPPORTED;
    return PG_ERR_CUDA;
}

// ordered: one group per key with no wrap-around (a region-ordered batch), so
// the resident blocks always cover one contiguous window of the batch
void launch_shape(const pg_table *t, uint32_t lanes, uint64_t n, dim3 &grid, dim3 &block, bool ordered = false)
{
    const uint32_t bt = t->block_threads;
    const uint64_t groups_per_block = bt / lanes;
    uint64_t need = (n + groups_per_block - 1) / groups_per_block;
    uint64_t cap = ordered ? 0x7fffffffull : (uint64_t)t->num_sms * t->blocks_per_sm;
    if (t->max_blocks && cap > t->max_blocks) cap = t->max_blocks;
    if (need > cap) need = cap;
    if (need == 0) need = 1;
    grid = dim3((unsigned)need);
    block = dim3(bt);
}

pg_status run_bulk(pg_table *t, int op, const bulk_args &a, pg_stream_t stream)
{
    if (!t || !pg_on_device(t->device)) return PG_ERR_INVALID;
    if (a.n == 0) return PG_OK;
    if (!a.keys) return PG_ERR_INVALID;
    dim3 grid, block;
    const uint32_t tile = pg_table_lanes(t, op);
    launch_shape(t, tile, a.n, grid, block, a.perm != nullptr);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t b0 = t->cfg.levels[0].bucket_size;
    const table_desc &d = t->desc;
    cudaError_t e;
    switch (t->ifmt) {
    case FMT_KV64: e = launch_kv64(op, b0, tile, d, a, grid, block, s); break;
    case FMT_KV64_SPLIT: e = launch_kv64_split(op, b0, tile, d, a, grid, block, s); break;
    case FMT_TAGVAL16: e = launch_tagval16(op, b0, tile, d, a, grid, block, s); break;
    case FMT_TAGVAL16_SPLIT: e = launch_tagval16_split(op, b0, tile, d, a, grid, block, s); break;
    case FMT_KV64_FP: e = launch_kv64_fp(op, b0, tile, d, a, grid, block, s); break;
    default: e = launch_tag16(op, b0, tile, d, a, grid, block, s); break;
    }
    return cuda_status(e);
}

// the bucketed filter's operations (packed formats)
pg_status run_packed(pg_table *t, int op, const packed_args &a, pg_stream_t stream)
{
    if (!t || !pg_on_device(t->device)) return PG_ERR_INVALID;
    if (t->ifmt != FMT_PACKED16 && t->ifmt != FMT_PACKED8) return PG_ERR_UNSUPPORTED;
    if (a.n == 0) return PG_OK;
    if (!a.keys) return PG_ERR_INVALID;
    // one group per key, blocks in batch order like the reference's one-tile-per-key
    // launch: with deletes in the mix, which of two keys sharing a tag holds the
    // earlier slot (and so which one a remove takes) follows the batch order
    const uint32_t lanes = pg_table_lanes(t, op);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t b0 = t->cfg.levels[0].bucket_size, b1 = t->cfg.nlevels > 1 ? t->cfg.levels[1].bucket_size : 8;
    // The insert forms into a two-choice primary level with fewer buckets than
    // the GPU holds keys at once run in launches of one key per bucket: with the
    // whole batch in flight together, every key's shortcut would see the fills
    // from before the batch and keys would pile into their first choices (a
    // 2^14-slot filter with 2 % backing filled to 0.9 failed ~340 keys in one
    // launch; the sequential order fails none).  Larger levels are unaffected.
    const bool inserts = op == POP_INSERT || op == POP_INSERT_DELETE || op == POP_INSERT_IF_NOT_EXISTS ||
                         op == POP_INSERT_IF_NOT_EXISTS_DELETE;
    const uint64_t nb0 = t->desc.lv[0].nbmod.d;
    const uint64_t resident = (uint64_t)t->num_sms * 2048;
    const uint64_t chunk = inserts && t->cfg.levels[0].scheme == PG_SCHEME_TWO_CHOICE_BUCKETED && nb0 < resident &&
                                   t->max_blocks != 1
                               ? nb0
                               : a.n;
    const uint32_t vb = t->ifmt == FMT_PACKED16 ? 2u : 1u;
    for (uint64_t off = 0; off < a.n; off += chunk) {
        packed_args c = a;
        c.n = a.n - off < chunk ? a.n - off : chunk;
        c.keys = a.keys + off;
        if (a.vals_in) c.vals_in = static_cast<const unsigned char *>(a.vals_in) + off * vb;
        if (a.vals_out) c.vals_out = static_cast<unsigned char *>(a.vals_out) + off * vb;
        if (a.flags) c.flags = a.flags + off;
        if (a.found) c.found = a.found + off;
        dim3 grid, block;
        launch_shape(t, lanes, c.n, grid, block, true);
        const cudaError_t e = t->ifmt == FMT_PACKED16 ? launch_packed16(op, b0, b1, lanes, t->desc, c, grid, block, s)
                                                      : launch_packed8(op, b0, b1, lanes, t->desc, c, grid, block, s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    return PG_OK;
}

// occupied / tombstone counts of one level: one thread per bucket
template <class K>
__global__ void __launch_bounds__(256) k_count_fill(const unsigned char *base, uint64_t nb, uint32_t B,
                                                    uint32_t bucket_bytes, uint32_t key_stride, K tomb,
                                                    unsigned long long *out)
{
    uint32_t occ = 0, tmb = 0;
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned char *bk = base + b * bucket_bytes;
        for (uint32_t s = 0; s < B; s++) {
            K v = __ldcs(reinterpret_cast<const K *>(bk + s * key_stride));
            occ += v != (K)0;
            tmb += v == tomb;
        }
    }
    __shared__ unsigned int sh[2];
    if (threadIdx.x == 0) sh[0] = sh[1] = 0;
    __syncthreads();
    unsigned am = __activemask();
    unsigned so = __reduce_add_sync(am, occ), st = __reduce_add_sync(am, tmb);
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(&sh[0], so);
        atomicAdd(&sh[1], st);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (sh[0]) atomicAdd(out, (unsigned long long)sh[0]);
        if (sh[1]) atomicAdd(out + 1, (unsigned long long)sh[1]);
    }
}

// fingerprint bytes recomputed from the slots (after a level is loaded)
__global__ void __launch_bounds__(256) k_rebuild_fp(const unsigned char *base, unsigned char *fp, uint64_t nslots,
                                                    uint64_t seed)
{
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t key = *reinterpret_cast<const unsigned long long *>(base + 16 * s);
        fp[s] = fp_of(key, murmur64a_u64(key, seed));
    }
}

}  // namespace

// Lanes per key for one operation.  Unless pg_table_set_launch fixed them,
// the fastest measured on B200 (2^22-2^30 slots, 0.85-0.9 load): one lane
// per key, which loads the whole bucket itself, except two for queries and
// removes of uint64 tables without fingerprints, whose 128-byte buckets two
// lanes scan faster (16.6 vs 10.1 G queries/s at 8-slot buckets; inserts
// 17.6 vs 13.0 G/s the other way).  The lanes never change a sequential
// result; they do change how many keys run at once.  Inserts into a
// two-choice level of fewer than 2^18 slots take 4 lanes, the reference's
// tile: at one lane the whole batch is in flight together, the shortcut's
// fill checks see stale counts and keys pile into their first choice (a
// 2^16-slot TCF with 1 % backing at 0.9 load failed ~800 keys at one lane,
// ~100 in the reference's own build, none at 4 lanes).
uint32_t pg_table_lanes(const pg_table *t, int op)
{
    if (t->ifmt == FMT_PACKED16 || t->ifmt == FMT_PACKED8) return t->lanes >= 4 ? 4u : 1u;  // compiled widths
    // the fingerprinted kernels serve one key per lane: a grid sized for more
    // lanes per key would launch blocks past the batch's end
    if (t->ifmt == FMT_KV64_FP) return 1u;
    if (t->lanes) return t->lanes;
    const pg_level_config &L0 = t->cfg.levels[0];
    if (op == OP_INSERT && L0.scheme == PG_SCHEME_TWO_CHOICE && L0.nslots < (1ull << 18) &&
        t->block_threads % 4 == 0 && L0.bucket_size >= 4)
        return 4u;
    const bool kv = t->ifmt == FMT_KV64 || t->ifmt == FMT_KV64_SPLIT;
    return kv && op != OP_INSERT && t->block_threads % 2 == 0 ? 2u : 1u;
}

extern "C" {

const char *pg_version(void) { return "poggers_b200 0.1 sm_100a"; }

const char *pg_status_string(pg_status s)
{
    switch (s) {
    case PG_OK: return "ok";
    case PG_ERR_INVALID: return "invalid argument";
    case PG_ERR_CUDA: return "CUDA error";
    case PG_ERR_NOMEM: return "out of device memory";
    case PG_ERR_UNSUPPORTED: return "unsupported configuration";
    case PG_ERR_FULL: return "capacity exhausted";
    case PG_ERR_TIMEOUT: return "bounded device wait timed out";
    case PG_ERR_TOO_LARGE:
        return "more tables or requests than pg_batch_run_static's fixed scratch holds "
               "(PG_STATIC_MAX_TABLES / PG_STATIC_MAX_OPS)";
    }
    return "unknown status";
}

pg_status pg_table_create(const pg_table_config *cfg, uint64_t seed, pg_table **out)
{
    if (!out) return PG_ERR_INVALID;
    *out = nullptr;
    pg_status st = validate(cfg);
    if (st != PG_OK) return st;
    pg_table *t = (pg_table *)calloc(1, sizeof(pg_table));
    if (!t) return PG_ERR_NOMEM;
    t->cfg = *cfg;
    if (cudaGetDevice(&t->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, t->device) != cudaSuccess) {
        free(t);
        return PG_ERR_CUDA;
    }
    t->block_threads = 256;
    t->blocks_per_sm = 32;
    t->max_blocks = 0;
    // lanes per key chosen per operation (pg_table_lanes) until set_launch fixes them
    t->lanes = 0;
    t->partition = 1;
    t->ifmt = internal_format(cfg);
    t->desc.nlevels = cfg->nlevels;
    t->desc.format = t->ifmt;
    const uint32_t kb = key_bytes(cfg->format), vb = val_bytes(cfg->format);
    uint64_t s = seed;
    for (uint32_t l = 0; l < cfg->nlevels; l++) {
        const pg_level_config &L = cfg->levels[l];
        level_desc &D = t->desc.lv[l];
        const uint64_t nb = (L.nslots - 1) / L.bucket_size + 1;  // min_buckets, bucket_insert.cuh:90
        D.bucket_size = L.bucket_size;
        D.max_probes = L.max_probes;
        D.scheme = L.scheme;
        D.probe = L.probe;
        D.bucket_bytes = L.bucket_size * (kb + vb);
        D.nbmod = make_fastmod64(nb);
        D.seed = s;
        D.seed2 = s * s;
        t->bytes[l] = nb * D.bucket_bytes;
        cudaError_t e = cudaMalloc(&t->mem[l], t->bytes[l]);
        if (e == cudaSuccess) e = cudaMemset(t->mem[l], 0, t->bytes[l]);
        if (e != cudaSuccess) {
            cudaGetLastError();
            for (uint32_t j = 0; j <= l; j++)
                if (t->mem[j]) cudaFree(t->mem[j]);
            free(t);
            return cuda_status(e);
        }
        D.base = static_cast<unsigned char *>(t->mem[l]);
        D.fp = nullptr;
        if (l == 0 && fingerprinted(cfg)) {
            t->fp_bytes = nb * L.bucket_size;
            e = cudaMalloc(&t->fp, t->fp_bytes);
            if (e == cudaSuccess) e = cudaMemset(t->fp, 0, t->fp_bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                pg_table_destroy(t);
                return cuda_status(e);
            }
            D.fp = static_cast<unsigned char *>(t->fp);
            D.fp_resident = t->fp_bytes <= kFpResidentBytes;
        }
        s = s * s;  // recursive table gets seed*seed (base_table.cuh:124)
    }
    *out = t;
    return PG_OK;
}

pg_status pg_table_destroy(pg_table *t)
{
    if (!t) return PG_ERR_INVALID;
    pg_status st = PG_OK;
    for (int l = 0; l < 2; l++)
        if (t->mem[l] && cudaFree(t->mem[l]) != cudaSuccess) st = PG_ERR_CUDA;
    if (t->fp && cudaFree(t->fp) != cudaSuccess) st = PG_ERR_CUDA;
    if (t->part_buf && cudaFree(t->part_buf) != cudaSuccess) st = PG_ERR_CUDA;
    free(t);
    return st;
}

pg_status pg_table_clear(pg_table *t, pg_stream_t stream)
{
    if (!t || !pg_on_device(t->device)) return PG_ERR_INVALID;
    for (uint32_t l = 0; l < t->cfg.nlevels; l++) {
        cudaError_t e = cudaMemsetAsync(t->mem[l], 0, t->bytes[l], reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_status(e);
    }
    if (t->fp) return cuda_status(cudaMemsetAsync(t->fp, 0, t->fp_bytes, reinterpret_cast<cudaStream_t>(stream)));
    return PG_OK;
}

pg_status pg_table_level_info(const pg_table *t, uint32_t level, pg_level_info *out)
{
    if (!t || !out || level >= t->cfg.nlevels) return PG_ERR_INVALID;
    const level_desc &D = t->desc.lv[level];
    out->nbuckets = D.nbmod.d;
    out->nslots = D.nbmod.d * D.bucket_size;
    out->bytes = t->bytes[level];
    out->seed = D.seed;
    out->d_buckets = t->mem[level];
    return PG_OK;
}

uint64_t pg_table_bytes(const pg_table *t)
{
    if (!t) return 0;
    return t->bytes[0] + t->bytes[1] + t->fp_bytes + t->part_bytes;
}

pg_status pg_table_set_partitioned_insert(pg_table *t, int enable)
{
    if (!t) return PG_ERR_INVALID;
    t->partition = enable != 0;
    return PG_OK;
}

pg_status pg_table_set_fingerprint_residency(pg_table *t, int resident)
{
    if (!t || !t->fp) return PG_ERR_INVALID;
    t->desc.lv[0].fp_resident = resident != 0;
    return PG_OK;
}

pg_status pg_table_reserve_insert_scratch(pg_table *t, uint64_t max_batch_keys, pg_stream_t stream)
{
    if (!t || !pg_on_device(t->device)) return PG_ERR_INVALID;
    return pg_partition_reserve(t, max_batch_keys, reinterpret_cast<cudaStream_t>(stream)) ? PG_OK : PG_ERR_NOMEM;
}

pg_status pg_table_set_launch(pg_table *t, uint32_t block_threads, uint32_t blocks_per_sm, uint32_t max_blocks,
                              uint32_t lanes_per_key)
{
    if (!t) return PG_ERR_INVALID;
    if (!(lanes_per_key == 0 || lanes_per_key == 1 || lanes_per_key == 2 || lanes_per_key == 4 ||
          lanes_per_key == 8 || lanes_per_key == 16))
        return PG_ERR_INVALID;
    if (lanes_per_key > t->cfg.levels[0].bucket_size) return PG_ERR_UNSUPPORTED;
    if (block_threads == 0) block_threads = 256;
    if (blocks_per_sm == 0) blocks_per_sm = 32;
    if (block_threads > 256 || (lanes_per_key && block_threads % lanes_per_key != 0)) return PG_ERR_INVALID;
    if (block_threads < 32 && max_blocks != 1) return PG_ERR_INVALID;  // partial warps only for the serial shape
    t->lanes = lanes_per_key;
    t->block_threads = block_threads;
    t->blocks_per_sm = blocks_per_sm;
    t->max_blocks = max_blocks;
    return PG_OK;
}

pg_status pg_bulk_insert(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n, uint8_t *d_ok,
                         uint64_t *d_fail_count, pg_stream_t stream)
{
    if (t && packed(t->cfg.format)) {
        packed_args p{d_keys, d_vals, nullptr, d_ok, nullptr, reinterpret_cast<unsigned long long *>(d_fail_count), n};
        return run_packed(t, POP_INSERT, p, stream);
    }
    if (t && !pg_on_device(t->device)) return PG_ERR_INVALID;  // before the region sort launches anything
    bulk_args a{d_keys, t && t->cfg.format != PG_FMT_TAG16 ? d_vals : nullptr, nullptr, d_ok,
                reinterpret_cast<unsigned long long *>(d_fail_count), n};
    const bulk_args batch = a;
    const uint32_t *only = nullptr;
    if (t && d_keys && n && pg_partition_insert(t, a, only, reinterpret_cast<cudaStream_t>(stream))) {
        // the sorted runs, then any keys that did not fit their run
        const pg_status st = run_bulk(t, OP_INSERT, a, stream);
        if (st != PG_OK) return st;
        bulk_args rest = batch;
        rest.only = only;
        return run_bulk(t, OP_INSERT, rest, stream);
    }
    return run_bulk(t, OP_INSERT, a, stream);
}

pg_status pg_bulk_query(pg_table *t, const uint64_t *d_keys, uint64_t n, void *d_vals_out, uint8_t *d_found,
                        uint64_t *d_hit_count, pg_stream_t stream)
{
    if (t && packed(t->cfg.format)) {
        packed_args p{d_keys, nullptr, d_vals_out, d_found, nullptr, reinterpret_cast<unsigned long long *>(d_hit_count),
                      n};
        return run_packed(t, POP_QUERY, p, stream);
    }
    bulk_args a{d_keys, nullptr, d_vals_out, d_found, reinterpret_cast<unsigned long long *>(d_hit_count), n};
    return run_bulk(t, OP_QUERY, a, stream);
}

pg_status pg_bulk_remove(pg_table *t, const uint64_t *d_keys, uint64_t n, uint8_t *d_ok, uint64_t *d_hit_count,
                         pg_stream_t stream)
{
    if (t && packed(t->cfg.format)) {
        packed_args p{d_keys, nullptr, nullptr, d_ok, nullptr, reinterpret_cast<unsigned long long *>(d_hit_count), n};
        return run_packed(t, POP_REMOVE, p, stream);
    }
    bulk_args a{d_keys, nullptr, nullptr, d_ok, reinterpret_cast<unsigned long long *>(d_hit_count), n};
    return run_bulk(t, OP_REMOVE, a, stream);
}

pg_status pg_bulk_insert_with_delete(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n,
                                     uint8_t *d_ok, uint64_t *d_fail_count, pg_stream_t stream)
{
    packed_args p{d_keys, d_vals, nullptr, d_ok, nullptr, reinterpret_cast<unsigned long long *>(d_fail_count), n};
    return run_packed(t, POP_INSERT_DELETE, p, stream);
}

pg_status pg_bulk_insert_if_not_exists(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n,
                                       void *d_vals_out, uint8_t *d_found, uint8_t *d_ok, uint64_t *d_fail_count,
                                       pg_stream_t stream)
{
    packed_args p{d_keys, d_vals, d_vals_out, d_ok, d_found, reinterpret_cast<unsigned long long *>(d_fail_count), n};
    return run_packed(t, POP_INSERT_IF_NOT_EXISTS, p, stream);
}

pg_status pg_bulk_insert_if_not_exists_delete(pg_table *t, const uint64_t *d_keys, const void *d_vals, uint64_t n,
                                              void *d_vals_out, uint8_t *d_found, uint8_t *d_ok,
                                              uint64_t *d_fail_count, pg_stream_t stream)
{
    packed_args p{d_keys, d_vals, d_vals_out, d_ok, d_found, reinterpret_cast<unsigned long long *>(d_fail_count), n};
    return run_packed(t, POP_INSERT_IF_NOT_EXISTS_DELETE, p, stream);
}

pg_status pg_table_count_fill(pg_table *t, uint32_t level, uint64_t *d_out, pg_stream_t stream)
{
    if (!t || !d_out || level >= t->cfg.nlevels || !pg_on_device(t->device)) return PG_ERR_INVALID;
    const level_desc &D = t->desc.lv[level];
    const uint64_t nb = D.nbmod.d;
    uint64_t blocks = (nb + 255) / 256;
    uint64_t cap = (uint64_t)t->num_sms * 8;
    if (blocks > cap) blocks = cap;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    auto *out = reinterpret_cast<unsigned long long *>(d_out);
    // keys sit every key_bytes (split layout, tag-only) or every slot (interleaved)
    const uint32_t stride = split_layout(&t->cfg) ? key_bytes(t->cfg.format)
                                                  : key_bytes(t->cfg.format) + val_bytes(t->cfg.format);
    if (t->cfg.format == PG_FMT_KV64)
        k_count_fill<unsigned long long><<<(unsigned)blocks, 256, 0, s>>>(D.base, nb, D.bucket_size, D.bucket_bytes,
                                                                          stride, ~0ULL, out);
    else if (t->cfg.format == PG_FMT_PACKED_TAGVAL16)  // whole words; the tombstone word is tag 0xFFFF, value 0
        k_count_fill<unsigned int><<<(unsigned)blocks, 256, 0, s>>>(D.base, nb, D.bucket_size, D.bucket_bytes, 4u,
                                                                    0xFFFFu, out);
    else if (t->cfg.format == PG_FMT_PACKED_TAGVAL8)
        k_count_fill<unsigned short><<<(unsigned)blocks, 256, 0, s>>>(D.base, nb, D.bucket_size, D.bucket_bytes, 2u,
                                                                      (unsigned short)0x00FFu, out);
    else
        k_count_fill<unsigned short><<<(unsigned)blocks, 256, 0, s>>>(D.base, nb, D.bucket_size, D.bucket_bytes,
                                                                      stride, (unsigned short)0xFFFFu, out);
    return cuda_status(cudaGetLastError());
}

// Reference slot layout: slot s of bucket b at (b*B + s) * slot_bytes, the
// key first, then the val (key_val_pair.cuh:72-74); tag-only slots hold the
// key.  The interleaved layout is that layout already; the split layout is a
// per-bucket permutation of it.
pg_status pg_table_dump_level(const pg_table *t, uint32_t level, void *host_dst, uint64_t bytes)
{
    if (!t || !host_dst || level >= t->cfg.nlevels) return PG_ERR_INVALID;
    const level_desc &D = t->desc.lv[level];
    const uint32_t kb = key_bytes(t->cfg.format), vb = val_bytes(t->cfg.format), sb = kb + vb;
    const uint64_t nslots = D.nbmod.d * D.bucket_size;
    if (bytes != nslots * sb) return PG_ERR_INVALID;
    if (!split_layout(&t->cfg))
        return cuda_status(cudaMemcpy(host_dst, t->mem[level], t->bytes[level], cudaMemcpyDeviceToHost));
    std::vector<unsigned char> raw(t->bytes[level]);
    cudaError_t e = cudaMemcpy(raw.data(), t->mem[level], t->bytes[level], cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e);
    unsigned char *dst = static_cast<unsigned char *>(host_dst);
    const uint32_t B = D.bucket_size;
    for (uint64_t b = 0; b < D.nbmod.d; b++) {
        const unsigned char *src = raw.data() + b * D.bucket_bytes;
        for (uint32_t s = 0; s < B; s++) {
            unsigned char *slot = dst + (b * B + s) * sb;
            memcpy(slot, src + s * kb, kb);
            memcpy(slot + kb, src + B * kb + s * vb, vb);
        }
    }
    return PG_OK;
}

pg_status pg_table_load_level(pg_table *t, uint32_t level, const void *host_src, uint64_t bytes)
{
    // a fingerprinted level's index is rebuilt by a kernel on the table's device
    if (!t || !host_src || level >= t->cfg.nlevels || !pg_on_device(t->device)) return PG_ERR_INVALID;
    const level_desc &D = t->desc.lv[level];
    const uint32_t kb = key_bytes(t->cfg.format), vb = val_bytes(t->cfg.format), sb = kb + vb;
    const uint64_t nslots = D.nbmod.d * D.bucket_size;
    if (bytes != nslots * sb) return PG_ERR_INVALID;
    if (!split_layout(&t->cfg)) {
        cudaError_t e = cudaMemcpy(t->mem[level], host_src, t->bytes[level], cudaMemcpyHostToDevice);
        if (e == cudaSuccess && level == 0 && t->fp) {
            k_rebuild_fp<<<1184, 256>>>(D.base, D.fp, nslots, D.seed);
            e = cudaDeviceSynchronize();
        }
        return cuda_status(e);
    }
    std::vector<unsigned char> raw(t->bytes[level]);
    const unsigned char *src = static_cast<const unsigned char *>(host_src);
    const uint32_t B = D.bucket_size;
    for (uint64_t b = 0; b < D.nbmod.d; b++) {
        unsigned char *dst = raw.data() + b * D.bucket_bytes;
        for (uint32_t s = 0; s < B; s++) {
            const unsigned char *slot = src + (b * B + s) * sb;
            memcpy(dst + s * kb, slot, kb);
            memcpy(dst + B * kb + s * vb, slot + kb, vb);
        }
    }
    return cuda_status(cudaMemcpy(t->mem[level], raw.data(), t->bytes[level], cudaMemcpyHostToDevice));
}

uint64_t pg_host_murmur64a(uint64_t key, uint64_t seed) { return murmur64a_u64(key, seed); }

uint64_t pg_host_fastmod(uint64_t n, uint64_t d)
{
    if (d == 0) return 0;
    return make_fastmod64(d).mod(n);
}

uint32_t pg_host_probe_buckets(const pg_table_config *cfg, uint32_t level, uint64_t seed, uint64_t key, uint64_t *out,
                               uint32_t cap)
{
    if (validate(cfg) != PG_OK || level >= cfg->nlevels || !out) return 0;
    uint64_t s = seed;
    for (uint32_t l = 0; l < level; l++) s = s * s;
    const pg_level_config &L = cfg->levels[level];
    const uint64_t nb = (L.nslots - 1) / L.bucket_size + 1;
    const fastmod64 fm = make_fastmod64(nb);
    const uint64_t tag = cfg->format == PG_FMT_KV64 ? key : tag16(key);
    probe_seq ps;
    ps.begin(L.probe, key, tag, s, s * s);
    uint32_t n = 0;
    for (uint32_t i = 0; i < L.max_probes && n < cap; i++) {
        uint64_t raw = ps.at(i);
        if (raw == kProbeEnd) break;
        out[n++] = fm.mod(raw);
    }
    return n;
}

}  // extern "C"
