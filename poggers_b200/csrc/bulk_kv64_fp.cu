// bulk_kv64_fp.cu -- bulk kernels for uint64 tables with a fingerprint index
// (one lane per key, bucket_insert primary level; see level_ops_fp).
#include <mutex>

#include "bulk_kernels.cuh"

namespace pg {

// Query with lane refill.  A negative query walks a variable number of
// buckets (1 to max_probes), and with one key per lane a warp would run as
// long as its slowest lane while the others idle.  Here every warp owns a
// contiguous range of the batch and runs probe steps: in each step every
// active lane does one bucket of its key, and a lane whose key is resolved
// takes the next key of the warp's range, so the warp's lanes stay busy until
// the range is exhausted.  The per-key rule is level_ops_fp::query_s exactly
// (first fingerprint match at or before the first empty slot of a bucket,
// a bucket with an empty slot ends the walk); a primary miss goes to the
// backing level.
// While the fingerprint array stays in L2 (level_desc::fp_resident), each
// step reads the fingerprint words of two consecutive probes of a key: an
// absent key walks about 2.9 buckets at 0.9 load, so its chain of dependent
// L2 round trips halves.  Measured at 2^26 slots: query 2.041 ms against
// 2.078 reading one bucket per step (45 registers against 32).  A larger
// array is read from DRAM, where the second word read is a second random
// access for every key: at 2^30 slots (1 GiB of fingerprints) the query
// took 66.2 ms reading two buckets per step against 52.6 reading one.
// Build knob: 0 = one bucket per step always, 1 = two while resident, 2 = two always.
#ifndef PG_FP_QUERY_TWO_MODE
#define PG_FP_QUERY_TWO_MODE 1
#endif

// Reading two buckets per step, held to 6 resident blocks of 256 (40
// registers, a word spilled) the kernel ran 1.913 ms against 2.030 at its
// natural 46 registers (5 blocks) at 2^26 slots; 8 blocks (32 registers)
// 2.26 ms.  Dealing each block's range to its warps in 128-key chunks from a
// shared counter (so that no warp idles at the end of a fixed range) measured
// 1.934 ms at 6 blocks: not kept.  Reading one bucket per step it fits 32
// registers, full occupancy.
#ifndef PG_FP_QUERY_MIN_BLOCKS
#define PG_FP_QUERY_MIN_BLOCKS 6
#endif

template <int B, bool BK, bool TWO>
__global__ void __launch_bounds__(256, TWO ? PG_FP_QUERY_MIN_BLOCKS : 8) k_query_fp_refill(table_desc t, bulk_args a)
{
    using P = level_ops_fp<B>;
    using BKO = backing_ops<FMT_KV64, 1>;
    constexpr int NW = P::NW;
    const level_desc &L = t.lv[0];
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t per = (a.n + nwarps - 1) / nwarps;
    uint64_t cursor = warp * per;
    const uint64_t end = cursor + per < a.n ? cursor + per : a.n;
    const uint64_t keep = fp_policy(L), stream = l2_policy_evict_first();
    unsigned long long *vout = static_cast<unsigned long long *>(a.vals_out);
    const uint32_t lt = (1u << lane) - 1u;
    bool active = false;
    uint64_t idx = 0, key = 0;
    uint32_t f = 0, i = 0;
    probe_seq ps;
    uint32_t hits = 0;
    while (true) {
        // refill: lanes without a key take the next keys of the range, in lane order
        const uint32_t need = __ballot_sync(0xffffffffu, !active);
        if (need) {
            const uint64_t mine = cursor + __popc(need & lt);
            cursor += __popc(need);
            if (!active && mine < end) {
                active = true;
                idx = mine;
                key = __ldcs(a.keys + idx);
                ps.begin(L.probe, key, key, L.seed, L.seed2);
                f = fp_of(key, ps.h1);
                i = 0;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active) {
            // one bucket of this lane's key (two with TWO: the next
            // probe's fingerprints are read with this one's and looked at only
            // if the walk goes on, so the results are the same)
            bool done = false, hit = false;
            unsigned long long v = 0;
            const uint64_t raw = ps.at(i);
            if (raw == kProbeEnd) {
                done = true;
            } else {
                const uint64_t b = L.nbmod.mod(raw);
                uint32_t w[NW], w2[NW];
                P::load_fp(L, b, w, keep);
                uint64_t b2 = 0;
                bool two = false;
                if constexpr (TWO) {
                    if (i + 1 < L.max_probes) {
                        const uint64_t raw2 = ps.at(i + 1);
                        if (raw2 != kProbeEnd) {
                            two = true;
                            b2 = L.nbmod.mod(raw2);
                            P::load_fp(L, b2, w2, keep);
                        }
                    }
                }
                // a bucket's rule: first fingerprint match at or before its first empty slot
                auto look = [&](uint64_t bb, const uint32_t (&ww)[NW]) -> uint32_t {
                    const uint32_t e = P::match(ww, 0);
                    uint32_t cand = P::match(ww, f) & P::upto(e);
                    while (cand) {
                        const int sl = __ffs(cand) - 1;
                        unsigned long long k, vv;
                        P::load_slot(L, bb, sl, k, vv, stream);
                        if (k == key) {
                            hit = true;
                            v = vv;
                            break;
                        }
                        cand &= cand - 1;
                    }
                    return e;
                };
                uint32_t e = look(b, w);
                done = hit || e != 0 || ++i >= L.max_probes;
                if (TWO && !done && two) {
                    e = look(b2, w2);
                    done = hit || e != 0 || ++i >= L.max_probes;
                }
            }
            if (done) {
                if (!hit && BK && t.nlevels > 1) {
                    const group<1> g1 = group<1>::make();
                    hit = BKO::query(t.lv[1], g1, key, &v);
                }
                if (vout) __stcs(vout + idx, hit ? v : 0ULL);
                if (a.flags) __stcs(a.flags + idx, (uint8_t)hit);
                hits += hit;
                active = false;
            }
        }
    }
    add_count(a.count, hits);
}

// Region-ordered insert (the sorted runs of partition.cu), one thread per
// entry with blocks in batch order, so the resident blocks sweep the table
// region by region.  Each key tries its first probe; a key whose first bucket
// is full (about one in eight at 0.9 load) joins the block's queue, and once
// the block's first attempts are done its threads take the queued keys
// together, from their second probe on (then the backing level).  Without the
// queue a warp runs every later probe of its slowest lane with most lanes idle.
#ifndef PG_FP_INSERT_QUEUE
#define PG_FP_INSERT_QUEUE 1
#endif
template <int B, bool BK>
__global__ void __launch_bounds__(256, PG_FP_MIN_BLOCKS) k_insert_fp_runs(table_desc t, bulk_args a)
{
    using P = level_ops_fp<B>;
    using BKO = backing_ops<FMT_KV64, 1>;
    __shared__ uint32_t queue[256];
    __shared__ uint32_t qn;
    if (threadIdx.x == 0) qn = 0;
    __syncthreads();
    const level_desc &L = t.lv[0];
    const unsigned long long *vin = static_cast<const unsigned long long *>(a.vals_in);
    const uint64_t base = (uint64_t)blockIdx.x * blockDim.x;
    const uint64_t i = base + threadIdx.x;
    bool live = i < a.n;
    if (live) {
        // past the keys of this region's run: nothing there
        const uint64_t r = __umul64hi(a.region_div, i);
        live = i - r * a.region_cap < a.region_cursor[r] - r * a.region_cap;
    }
    if (live) {
        const uint64_t key = __ldg(a.keys + i);
        const unsigned long long v = vin ? __ldg(vin + i) : 0ULL;
        if (!P::insert_probes(L, key, v, 0, 1)) queue[atomicAdd(&qn, 1u)] = threadIdx.x;
    }
    __syncthreads();
    const uint32_t nq = qn;
    uint32_t fails = 0;
    for (uint32_t q = threadIdx.x; q < nq; q += blockDim.x) {
        const uint64_t j = base + queue[q];
        const uint64_t key = __ldg(a.keys + j);
        const unsigned long long v = vin ? __ldg(vin + j) : 0ULL;
        bool r = P::insert_probes(L, key, v, 1, L.max_probes);
        if (!r && BK && t.nlevels > 1) r = BKO::insert(t.lv[1], group<1>::make(), key, v);
        if (!r) {
            if (a.flags) a.flags[a.perm[j]] = 0;
            fails++;
        }
    }
    add_count(a.count, fails);
}

// resident 256-thread blocks of a kernel on the current device (0 if unknown);
// looked up once per (device, kernel), under a lock so host threads may launch
// concurrently
int refill_blocks(const void *fn)
{
    struct entry {
        const void *fn;
        int dev, blocks;
    };
    static std::mutex mu;
    static entry cache[32];
    static int used = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    std::lock_guard<std::mutex> g(mu);
    for (int k = 0; k < used; ++k)
        if (cache[k].fn == fn && cache[k].dev == dev) return cache[k].blocks;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0) != cudaSuccess || per_sm <= 0) {
        cudaGetLastError();
        return 0;
    }
    if (used < 32) cache[used++] = entry{fn, dev, sms * per_sm};
    return sms * per_sm;
}

template <int B, bool BK, bool TWO>
cudaError_t launch_query_refill_k(const table_desc &t, const bulk_args &a, dim3 grid, cudaStream_t s)
{
    const void *fn = (const void *)k_query_fp_refill<B, BK, TWO>;
    const int blocks = refill_blocks(fn);
    // one resident wave of blocks, never more warps than keys
    uint64_t g = blocks > 0 ? (uint64_t)blocks : grid.x;
    const uint64_t max_by_keys = (a.n + 255) / 256;
    if (g > max_by_keys) g = max_by_keys;
    if (g < 1) g = 1;
    k_query_fp_refill<B, BK, TWO><<<(unsigned)g, 256, 0, s>>>(t, a);
    return cudaGetLastError();
}

template <int B, bool BK>
cudaError_t launch_query_refill(const table_desc &t, const bulk_args &a, dim3 grid, cudaStream_t s)
{
    const bool two = PG_FP_QUERY_TWO_MODE == 2 || (PG_FP_QUERY_TWO_MODE == 1 && t.lv[0].fp_resident);
    return two ? launch_query_refill_k<B, BK, true>(t, a, grid, s) : launch_query_refill_k<B, BK, false>(t, a, grid, s);
}

template <int B>
cudaError_t launch_fp_b(int op, const table_desc &t, const bulk_args &a, dim3 grid, dim3 block, cudaStream_t s)
{
    const bool bk = t.nlevels > 1;
    // the sorted runs of a region-ordered insert (one thread per entry; see k_insert_fp_runs)
    if (PG_FP_INSERT_QUEUE && op == OP_INSERT && a.region_cap && !a.only && block.x == 256 && a.perm) {
        const uint64_t blocks = (a.n + 255) / 256;
        if (bk) k_insert_fp_runs<B, true><<<(unsigned)blocks, 256, 0, s>>>(t, a);
        else k_insert_fp_runs<B, false><<<(unsigned)blocks, 256, 0, s>>>(t, a);
        return cudaGetLastError();
    }
    // the refill query needs whole warps; the serial shape (one lane) keeps the plain kernel
    if (op == OP_QUERY && block.x == 256 && grid.x > 1)
        return bk ? launch_query_refill<B, true>(t, a, grid, s) : launch_query_refill<B, false>(t, a, grid, s);
    return bk ? launch_bgs<FMT_KV64_FP, B, 1, SCHEME_BUCKET, true>(op, t, a, grid, block, s)
              : launch_bgs<FMT_KV64_FP, B, 1, SCHEME_BUCKET, false>(op, t, a, grid, block, s);
}

PG_DECLARE_LAUNCH(launch_kv64_fp)
{
    (void)tile;
    switch (bucket) {
    case 4: return launch_fp_b<4>(op, t, a, grid, block, s);
    case 8: return launch_fp_b<8>(op, t, a, grid, block, s);
    case 16: return launch_fp_b<16>(op, t, a, grid, block, s);
    case 32: return launch_fp_b<32>(op, t, a, grid, block, s);
    default: return cudaErrorInvalidConfiguration;
    }
}

}  // namespace pg
