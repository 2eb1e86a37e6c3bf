// batch.cu -- C ABI of the multi-table batch path (plan + persistent kernel).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime.h>

#include <mutex>

#include "poggers_b200.h"
#include "batch_kernels.cuh"
#include "table_internal.h"

using namespace pg;

struct pg_batch {
    uint32_t ntables;
    uint32_t max_ops;
    uint32_t ifmt, bucket, scheme;
    uint32_t bucket1;  // backing level's bucket size (the bucketed filter's kernels take it as a parameter)
    bool backing;
    table_desc *d_tables;
    // pg_batch_clear: the device ranges of every level and fingerprint array of
    // the batch's tables, and the running sum of their bytes
    uint32_t nseg;
    unsigned char **d_seg_ptr;
    unsigned long long *d_seg_bytes;
    unsigned long long *d_seg_end;  // inclusive prefix of the segments' spans rounded up to 16 bytes
    unsigned long long clear_padded;
    unsigned long long *d_scratch;  // chunk_start[max_ops + 1] then the work counter
    int num_sms;
    int device;  // the tables' device
    uint32_t block_threads, blocks_per_sm, lanes;
};

namespace pg {

__global__ void __launch_bounds__(1024) k_batch_plan(batch_args a)
{
    __shared__ unsigned long long carry;
    __shared__ unsigned long long warp_sums[32];
    uint32_t nops = *a.nops;
    if (nops > a.max_ops) nops = a.max_ops;
    if (threadIdx.x == 0) {
        carry = 0;
        *a.work = 0;
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < nops; base += blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        unsigned long long v = 0;
        if (j < nops) {
            const uint64_t ck = batch_chunk_keys(a, a.ops[j]);
            v = (a.ops[j].count + ck - 1) / ck;
        }
        // inclusive scan in the warp, then across warps
        unsigned long long x = v;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
            if ((int)lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
                if ((int)lane >= o) w += y;
            }
            warp_sums[lane] = w;  // inclusive prefix of warp totals
        }
        __syncthreads();
        const unsigned long long before = carry + (warp ? warp_sums[warp - 1] : 0) + x - v;
        if (j < nops) a.chunk_start[j] = before;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) a.chunk_start[nops] = carry;
}

// Zero every segment of a batch.  Each segment's span is rounded up to 16
// bytes in a global numbering (seg_end: inclusive prefix of the padded spans),
// so 16-byte chunk j lies inside one segment at an offset that is a multiple
// of 16; the segment is found by binary search, a full chunk is one 16-byte
// store (segment bases come from cudaMalloc, so they are aligned), and a
// segment's last partial chunk is written byte by byte, up to its true size.
__global__ void __launch_bounds__(256) k_batch_clear(unsigned char *const *seg, const unsigned long long *seg_bytes,
                                                     const unsigned long long *seg_end, uint32_t nseg,
                                                     unsigned long long padded_total)
{
    const unsigned long long chunks = padded_total / 16;
    for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < chunks;
         j += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long byte = j * 16;
        uint32_t lo = 0, hi = nseg - 1;  // first segment whose padded end is past `byte`
        while (lo < hi) {
            const uint32_t mid = (lo + hi) / 2;
            if (seg_end[mid] > byte) hi = mid;
            else lo = mid + 1;
        }
        const unsigned long long off = byte - (lo ? seg_end[lo - 1] : 0ULL);
        const unsigned long long n = seg_bytes[lo];
        if (off + 16 <= n) {
            *reinterpret_cast<uint4 *>(seg[lo] + off) = make_uint4(0, 0, 0, 0);
        } else {
            for (unsigned long long q = off; q < n; ++q) seg[lo][q] = 0;
        }
    }
}

}  // namespace pg

namespace {

// ---- scratch of pg_batch_run_static -------------------------------------
// For callers that cannot allocate device memory (code running where
// cudaMalloc is not available to it, e.g. inside another allocator, a
// driver-level plugin or an environment whose memory is fully budgeted), the
// batch run can use this fixed array instead of pg_batch_create's buffers.
// Every GPU that loads the library holds one copy until the process exits.
constexpr uint32_t kStaticMaxTables = PG_STATIC_MAX_TABLES;
constexpr uint32_t kStaticMaxOps = PG_STATIC_MAX_OPS;

struct static_scratch {
    table_desc tables[kStaticMaxTables];
    unsigned long long chunk_start[kStaticMaxOps + 1];
    unsigned long long work;
};

static __device__ __align__(256) unsigned char g_batch_static[sizeof(static_scratch)];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
// Device address of g_batch_static, per device ordinal, looked up once.  A
// cudaDeviceReset() frees the array with the context, so these addresses do not
// survive one: the entry point must not be used across a device reset.
void *g_static_addr[kMaxDevices];

// The descriptors reach the device array as kernel parameters (copied when the
// launch is enqueued), so no host buffer has to outlive the call.
constexpr uint32_t kStageChunk = 3840 / sizeof(table_desc);
static_assert(kStageChunk >= 1, "a table descriptor must fit in a kernel's parameters");
struct stage_chunk {
    table_desc d[kStageChunk];
};

__global__ void k_stage_tables(table_desc *dst, stage_chunk c, uint32_t n)
{
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = c.d[i];
}

// The symbol's device address on device `dev` (the current device); the first
// call on each device looks it up (cudaGetSymbolAddress, with that device current).
pg_status static_scratch_addr(int dev, static_scratch **out)
{
    if (dev < 0 || dev >= kMaxDevices) return PG_ERR_CUDA;
    if (!g_static_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_batch_static) != cudaSuccess || !p) {
            cudaGetLastError();
            return PG_ERR_CUDA;
        }
        g_static_addr[dev] = p;
    }
    *out = static_cast<static_scratch *>(g_static_addr[dev]);
    return PG_OK;
}

}  // namespace

namespace {

bool packed_fmt(uint32_t ifmt) { return ifmt == FMT_PACKED16 || ifmt == FMT_PACKED8; }

uint32_t backing_bucket(const pg_table *t) { return t->cfg.nlevels > 1 ? t->cfg.levels[1].bucket_size : 0; }

// one kernel instantiation serves a batch: same format, bucket, scheme and depth
// (and, for the bucketed filter, the same backing bucket size)
bool same_kernel(const pg_table *t, const pg_table *t0)
{
    return t && t->ifmt == t0->ifmt && t->cfg.levels[0].bucket_size == t0->cfg.levels[0].bucket_size &&
           t->cfg.levels[0].scheme == t0->cfg.levels[0].scheme && (t->cfg.nlevels > 1) == (t0->cfg.nlevels > 1) &&
           (!packed_fmt(t0->ifmt) || backing_bucket(t) == backing_bucket(t0)) && t->device == t0->device;
}

}  // namespace

extern "C" {

pg_status pg_batch_create(pg_table *const *tables, uint32_t ntables, uint32_t max_ops, pg_batch **out)
{
    if (!out || !tables || ntables == 0 || max_ops == 0) return PG_ERR_INVALID;
    *out = nullptr;
    const pg_table *t0 = tables[0];
    if (!t0) return PG_ERR_INVALID;
    for (uint32_t i = 1; i < ntables; i++) {
        const pg_table *t = tables[i];
        // one kernel instantiation serves the batch: same format, bucket, scheme and depth
        if (!same_kernel(t, t0)) return PG_ERR_UNSUPPORTED;
    }
    pg_batch *b = (pg_batch *)calloc(1, sizeof(pg_batch));
    if (!b) return PG_ERR_NOMEM;
    b->ntables = ntables;
    b->max_ops = max_ops;
    b->ifmt = t0->ifmt;
    b->bucket = t0->cfg.levels[0].bucket_size;
    b->scheme = t0->cfg.levels[0].scheme;
    b->backing = t0->cfg.nlevels > 1;
    b->bucket1 = backing_bucket(t0);
    b->num_sms = t0->num_sms;
    b->device = t0->device;
    b->block_threads = 256;
    b->blocks_per_sm = 8;
    b->lanes = pg_table_lanes(t0);
    table_desc *h = (table_desc *)malloc(sizeof(table_desc) * ntables);
    for (uint32_t i = 0; i < ntables; i++) h[i] = tables[i]->desc;
    // the ranges pg_batch_clear zeroes: what pg_table_clear zeroes, for every table
    const uint32_t maxseg = ntables * 3;
    unsigned char **sp = (unsigned char **)malloc(sizeof(unsigned char *) * maxseg);
    unsigned long long *sb = (unsigned long long *)malloc(sizeof(unsigned long long) * maxseg);
    unsigned long long *se = (unsigned long long *)malloc(sizeof(unsigned long long) * maxseg);
    uint32_t ns = 0;
    unsigned long long run = 0;
    auto add = [&](void *p, uint64_t bytes) {
        if (!p || !bytes) return;
        sp[ns] = static_cast<unsigned char *>(p);
        sb[ns] = bytes;
        run += (bytes + 15) / 16 * 16;
        se[ns++] = run;
    };
    for (uint32_t i = 0; i < ntables; i++) {
        for (uint32_t l = 0; l < tables[i]->cfg.nlevels; l++) add(tables[i]->mem[l], tables[i]->bytes[l]);
        add(tables[i]->fp, tables[i]->fp_bytes);
    }
    b->nseg = ns;
    b->clear_padded = run;
    cudaError_t e = cudaMalloc(&b->d_tables, sizeof(table_desc) * ntables);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_tables, h, sizeof(table_desc) * ntables, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_scratch, sizeof(unsigned long long) * ((uint64_t)max_ops + 2));
    if (e == cudaSuccess && ns) e = cudaMalloc(&b->d_seg_ptr, sizeof(unsigned char *) * ns);
    if (e == cudaSuccess && ns) e = cudaMalloc(&b->d_seg_bytes, sizeof(unsigned long long) * ns);
    if (e == cudaSuccess && ns) e = cudaMalloc(&b->d_seg_end, sizeof(unsigned long long) * ns);
    if (e == cudaSuccess && ns) e = cudaMemcpy(b->d_seg_ptr, sp, sizeof(unsigned char *) * ns, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ns) e = cudaMemcpy(b->d_seg_bytes, sb, sizeof(unsigned long long) * ns, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ns) e = cudaMemcpy(b->d_seg_end, se, sizeof(unsigned long long) * ns, cudaMemcpyHostToDevice);
    free(sp);
    free(sb);
    free(se);
    free(h);
    if (e != cudaSuccess) {
        cudaGetLastError();
        pg_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? PG_ERR_NOMEM : PG_ERR_CUDA;
    }
    *out = b;
    return PG_OK;
}

pg_status pg_batch_destroy(pg_batch *b)
{
    if (!b) return PG_ERR_INVALID;
    cudaFree(b->d_tables);
    cudaFree(b->d_scratch);
    cudaFree(b->d_seg_ptr);
    cudaFree(b->d_seg_bytes);
    cudaFree(b->d_seg_end);
    free(b);
    return PG_OK;
}

pg_status pg_batch_clear(pg_batch *b, pg_stream_t stream)
{
    if (!b || !pg_on_device(b->device)) return PG_ERR_INVALID;
    if (b->nseg == 0) return PG_OK;
    const unsigned long long chunks = b->clear_padded / 16;
    unsigned long long blocks = (chunks + 255) / 256;
    const unsigned long long cap = (unsigned long long)b->num_sms * 8;
    if (blocks > cap) blocks = cap;
    k_batch_clear<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        b->d_seg_ptr, b->d_seg_bytes, b->d_seg_end, b->nseg, b->clear_padded);
    return cudaGetLastError() == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

pg_status pg_batch_set_launch(pg_batch *b, uint32_t block_threads, uint32_t blocks_per_sm, uint32_t lanes_per_key)
{
    if (!b) return PG_ERR_INVALID;
    if (block_threads == 0) block_threads = 256;
    if (blocks_per_sm == 0) blocks_per_sm = 8;
    if (lanes_per_key == 0) lanes_per_key = b->lanes;
    if (b->ifmt == FMT_KV64_FP) lanes_per_key = 1;
    if (packed_fmt(b->ifmt)) lanes_per_key = lanes_per_key >= 4 ? 4 : 1;  // the widths built for the bucketed filter
    if (!(lanes_per_key == 1 || lanes_per_key == 2 || lanes_per_key == 4 || lanes_per_key == 8 ||
          lanes_per_key == 16) ||
        lanes_per_key > b->bucket)
        return PG_ERR_UNSUPPORTED;
    if (block_threads % 32 || block_threads > 256) return PG_ERR_INVALID;
    b->block_threads = block_threads;
    b->blocks_per_sm = blocks_per_sm;
    b->lanes = lanes_per_key;
    return PG_OK;
}

pg_status pg_batch_run(pg_batch *b, const pg_op_desc *d_ops, const uint32_t *d_nops, const uint64_t *d_keys,
                       const void *d_vals_in, void *d_vals_out, uint8_t *d_flags, uint64_t *d_op_counts,
                       pg_stream_t stream)
{
    if (!b || !d_ops || !d_nops || !d_keys || !pg_on_device(b->device)) return PG_ERR_INVALID;
    batch_args a;
    a.tables = b->d_tables;
    a.ops = d_ops;
    a.nops = d_nops;
    a.chunk_start = b->d_scratch;
    a.work = b->d_scratch + b->max_ops + 1;
    a.keys = d_keys;
    a.vals_in = d_vals_in;
    a.vals_out = d_vals_out;
    a.flags = d_flags;
    a.op_counts = reinterpret_cast<unsigned long long *>(d_op_counts);
    a.max_ops = b->max_ops;
    a.ntables = b->ntables;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_batch_plan<<<1, 1024, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return PG_ERR_CUDA;
    dim3 grid((unsigned)(b->num_sms * b->blocks_per_sm)), block(b->block_threads);
    const int sch = (int)b->scheme;
    switch (b->ifmt) {
    case FMT_KV64: e = batch_kv64(a, b->bucket, b->lanes, sch, b->backing, grid, block, s); break;
    case FMT_KV64_SPLIT: e = batch_kv64_split(a, b->bucket, b->lanes, sch, b->backing, grid, block, s); break;
    case FMT_TAGVAL16: e = batch_tagval16(a, b->bucket, b->lanes, sch, b->backing, grid, block, s); break;
    case FMT_TAGVAL16_SPLIT: e = batch_tagval16_split(a, b->bucket, b->lanes, sch, b->backing, grid, block, s); break;
    case FMT_KV64_FP: e = batch_kv64_fp(a, b->bucket, 1, sch, b->backing, grid, block, s); break;
    case FMT_PACKED16:
    case FMT_PACKED8: e = batch_packed(a, b->ifmt, b->bucket, b->bucket1, b->lanes, b->backing, grid, block, s); break;
    default: e = batch_tag16(a, b->bucket, b->lanes, sch, b->backing, grid, block, s); break;
    }
    if (e == cudaErrorInvalidConfiguration) return PG_ERR_UNSUPPORTED;
    return e == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

pg_status pg_batch_run_static(pg_table *const *tables, uint32_t ntables, const pg_op_desc *d_ops,
                              const uint32_t *d_nops, uint32_t max_ops, const uint64_t *d_keys,
                              const void *d_vals_in, void *d_vals_out, uint8_t *d_flags, uint64_t *d_op_counts,
                              pg_stream_t stream)
{
    if (!tables || ntables == 0 || !d_ops || !d_nops || !d_keys || max_ops == 0) return PG_ERR_INVALID;
    if (ntables > kStaticMaxTables || max_ops > kStaticMaxOps) return PG_ERR_TOO_LARGE;
    const pg_table *t0 = tables[0];
    if (!t0) return PG_ERR_INVALID;
    for (uint32_t i = 1; i < ntables; i++) {
        const pg_table *t = tables[i];
        if (!same_kernel(t, t0)) return PG_ERR_UNSUPPORTED;
    }
    // the array and the kernels live on the current device: it must be the tables'
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PG_ERR_CUDA;
    if (dev != t0->device) return PG_ERR_INVALID;
    std::lock_guard<std::mutex> g(g_static_mu);
    static_scratch *sc = nullptr;
    pg_status st = static_scratch_addr(dev, &sc);
    if (st != PG_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (uint32_t i = 0; i < ntables; i += kStageChunk) {
        const uint32_t m = ntables - i < kStageChunk ? ntables - i : kStageChunk;
        stage_chunk c;
        for (uint32_t j = 0; j < m; j++) c.d[j] = tables[i + j]->desc;
        k_stage_tables<<<1, 32, 0, s>>>(sc->tables + i, c, m);
        if (cudaGetLastError() != cudaSuccess) return PG_ERR_CUDA;
    }
    batch_args a;
    a.tables = sc->tables;
    a.ops = d_ops;
    a.nops = d_nops;
    a.chunk_start = sc->chunk_start;
    a.work = &sc->work;  // zeroed by k_batch_plan on every call
    a.keys = d_keys;
    a.vals_in = d_vals_in;
    a.vals_out = d_vals_out;
    a.flags = d_flags;
    a.op_counts = reinterpret_cast<unsigned long long *>(d_op_counts);
    a.max_ops = max_ops;
    a.ntables = ntables;
    k_batch_plan<<<1, 1024, 0, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return PG_ERR_CUDA;
    dim3 grid((unsigned)(t0->num_sms * 8)), block(256);
    const uint32_t lanes = pg_table_lanes(t0), bucket = t0->cfg.levels[0].bucket_size;
    const int sch = (int)t0->cfg.levels[0].scheme;
    const bool bk = t0->cfg.nlevels > 1;
    cudaError_t e;
    switch (t0->ifmt) {
    case FMT_KV64: e = batch_kv64(a, bucket, lanes, sch, bk, grid, block, s); break;
    case FMT_KV64_SPLIT: e = batch_kv64_split(a, bucket, lanes, sch, bk, grid, block, s); break;
    case FMT_TAGVAL16: e = batch_tagval16(a, bucket, lanes, sch, bk, grid, block, s); break;
    case FMT_TAGVAL16_SPLIT: e = batch_tagval16_split(a, bucket, lanes, sch, bk, grid, block, s); break;
    case FMT_KV64_FP: e = batch_kv64_fp(a, bucket, 1, sch, bk, grid, block, s); break;
    case FMT_PACKED16:
    case FMT_PACKED8: e = batch_packed(a, t0->ifmt, bucket, backing_bucket(t0), lanes, bk, grid, block, s); break;
    default: e = batch_tag16(a, bucket, lanes, sch, bk, grid, block, s); break;
    }
    if (e == cudaErrorInvalidConfiguration) return PG_ERR_UNSUPPORTED;
    return e == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}

}  // extern "C"
