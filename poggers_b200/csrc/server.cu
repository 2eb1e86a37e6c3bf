// server.cu -- continuous-batching server over resident tables.
//
// No counterpart in the reference.  Clients submit requests {table, op, keys,
// values} from host memory at any time; a worker thread packs the pending
// requests into "waves" and keeps up to kMaxWaves waves on the GPU at once:
// while one wave runs, the next is staged and launched behind it, so requests
// that arrive while others are on the GPU join the next wave instead of
// waiting for the queue to drain.  A wave is one pinned staging copy in (on
// the upload stream), one pg_batch_run per kernel class (tables of one format
// / bucket / scheme share a class), each on its class's own stream, and one
// copy out (on the download stream), ordered by events: the next wave's upload
// and the previous wave's download run beside this wave's kernels, and the
// classes of one wave run beside each other.
//
// Ordering: a class's runs are issued on its one stream in wave order, so
// requests on one table complete in submission order; and a wave never mixes
// conflicting requests on a table (only queries share a table with queries,
// inserts with inserts, removes with removes), so every result equals what the
// request returns when the requests are run one at a time in submission order
// (what the plain path does).
//
// Tables are admitted against an HBM budget: pg_server_add_table fails with
// PG_ERR_FULL when the table would not fit, and dropping a table releases its
// share.
#include <stdint.h>
#include <string.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <system_error>
#include <thread>
#include <vector>

#include "poggers_b200.h"
#include "table_internal.h"

namespace {

// Waves in flight, each with its own staging slot (pinned host and device
// buffers of about 31 bytes per key of max_wave_keys, outside the HBM
// budget).  Config 4 at 96 k / 128 k offered requests/s: p99 0.64-0.70 /
// 2.1-3.3 ms with 3 slots, 0.39-0.41 / 0.51-0.58 ms with 6, the same rates.
#ifndef PG_SERVER_WAVES
#define PG_SERVER_WAVES 6
#endif
constexpr int kMaxWaves = PG_SERVER_WAVES;

struct request {
    uint64_t id;
    uint32_t table;  // table id, or the slab set id when slab >= 0
    int32_t slab;    // -1: a table request; else PG_OP_MALLOC / PG_OP_FREE on slab set `table`
    uint32_t op;
    const uint64_t *keys;  // table keys; malloc: uint32_t sizes; free: object pointers
    const void *vals;
    uint64_t n;
    void *vals_out;
    uint8_t *flags;
    uint64_t count;  // hits or failures, filled on completion
    double t_submit, t_done;
};

struct table_entry {
    pg_table *t;
    uint32_t cls;      // kernel class
    uint32_t slot;     // index in its class's batch
    uint64_t bytes;
    bool live;
    uint32_t inflight = 0;  // requests taken into a wave and not yet completed
};

// a slab size-class set served by the loop: its requests run on its own stream
struct slab_entry {
    pg_slab_set *set = nullptr;
    cudaStream_t stream = nullptr;
    uint64_t bytes = 0;
    bool live = false;
    uint32_t inflight = 0;
};

struct klass {
    pg_batch *batch = nullptr;
    cudaStream_t stream = nullptr;  // the class's runs, in wave order
    std::vector<uint32_t> tables;  // server table ids in batch order
    uint32_t vbytes;
    bool dirty = true;  // batch must be rebuilt (tables added / dropped)
};

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct pg_server {
    pg_server_config cfg;
    int device;
    cudaStream_t stream;  // uploads
    cudaStream_t down;    // downloads
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t bytes_used = 0;
    std::vector<table_entry> tables;
    std::vector<klass> classes;
    std::vector<slab_entry> slabs;
    std::deque<request *> pending;
    std::map<uint64_t, request *> done;
    std::set<uint64_t> outstanding;  // submitted and not yet collected by pg_server_poll
    // staging (per wave slot): one pinned host buffer and one device buffer,
    // laid out per wave (wave_layout)
    struct stage {
        unsigned char *h, *d;
        cudaEvent_t uploaded;  // the wave's inputs are on the device
        cudaEvent_t ran;       // recorded after each class's run, waited on by the download stream
        cudaEvent_t done;
        bool busy;
    } stages[kMaxWaves];
    uint64_t waves_run = 0;
    uint64_t keys_run = 0;
    uint64_t requests_run = 0;
    // the worker thread's time by stage (seconds; written with the lock held)
    double t_plan = 0, t_copy_in = 0, t_issue = 0, t_copy_out = 0, t_wait_busy = 0, t_wait_idle = 0;
    pg_status error = PG_OK;
};

namespace {

uint32_t class_key(const pg_table *t)
{
    const bool packed = t->ifmt == pg::FMT_PACKED16 || t->ifmt == pg::FMT_PACKED8;
    const uint32_t b1 = packed && t->cfg.nlevels > 1 ? t->cfg.levels[1].bucket_size : 0u;
    return (t->ifmt << 24) | (b1 << 16) | (t->cfg.levels[0].bucket_size << 8) | (t->cfg.levels[0].scheme << 4) |
           (t->cfg.nlevels > 1 ? 1u : 0u);
}

bool conflicts(uint32_t a, uint32_t b) { return a != b; }

// staging buffer of a value width: 8 -> 0, 2 -> 1, 1 -> 2
int width_index(uint32_t vb) { return vb == 8 ? 0 : vb == 2 ? 1 : 2; }
constexpr uint32_t kWidths[3] = {8, 2, 1};

// Where one wave's inputs and outputs sit in its stage's buffers, at the same
// offsets on the host and on the device: the keys (a malloc's sizes and a
// free's pointers too), the values in by width, the requests, each class run's
// request count and the per-request counts are uploaded together, [0, up_end);
// the counts, the flags and the values out by width come back together,
// [counts, end).  Values are indexed like the keys; a width no request of the
// wave uses takes no room.
struct wave_layout {
    uint64_t keys, vin[3], ops, nops, counts, up_end, flags, vout[3], end;
    bool has_in[3], has_out[3];
};

uint64_t align16(uint64_t x) { return (x + 15) & ~15ull; }

wave_layout lay_out(uint64_t nkeys, uint64_t nreqs, uint64_t nruns, const bool in[3], const bool out[3])
{
    wave_layout L{};
    uint64_t at = 0;
    L.keys = at;
    at = align16(at + nkeys * 8);
    for (int x = 0; x < 3; x++) {
        L.has_in[x] = in[x];
        L.vin[x] = at;
        if (in[x]) at = align16(at + nkeys * kWidths[x]);
    }
    L.ops = at;
    at = align16(at + nreqs * sizeof(pg_op_desc));
    L.nops = at;
    at = align16(at + nruns * 4);
    L.counts = at;
    at = align16(at + nreqs * 8);
    L.up_end = at;
    L.flags = at;
    at = align16(at + nkeys);
    for (int x = 0; x < 3; x++) {
        L.has_out[x] = out[x];
        L.vout[x] = at;
        if (out[x]) at = align16(at + nkeys * kWidths[x]);
    }
    L.end = at;
    return L;
}

// wait for every wave the server has issued (uploads, every class's runs, downloads)
void sync_all(pg_server *s)
{
    cudaStreamSynchronize(s->stream);
    for (auto &k : s->classes)
        if (k.stream) cudaStreamSynchronize(k.stream);
    for (auto &e : s->slabs)
        if (e.stream) cudaStreamSynchronize(e.stream);
    cudaStreamSynchronize(s->down);
}

pg_status rebuild(pg_server *s, klass &k)
{
    if (k.batch) pg_batch_destroy(k.batch);
    k.batch = nullptr;
    std::vector<pg_table *> ts;
    for (uint32_t id : k.tables) {
        s->tables[id].slot = (uint32_t)ts.size();
        ts.push_back(s->tables[id].t);
    }
    if (!ts.empty()) {
        pg_status st = pg_batch_create(ts.data(), (uint32_t)ts.size(), s->cfg.max_wave_requests, &k.batch);
        if (st != PG_OK) return st;
        pg_batch_set_launch(k.batch, 256, 8, 0);
    }
    k.dirty = false;
    return PG_OK;
}

// Pack pending requests into stage `w` (caller holds the lock).  Returns the
// requests taken; the per-table order rule keeps results sequentially consistent.
std::vector<request *> take_wave(pg_server *s, pg_server::stage &st, uint64_t &nkeys, uint32_t &nops,
                                 std::vector<uint32_t> &ops_per_class)
{
    std::vector<request *> out;
    std::map<uint32_t, uint32_t> table_op;   // op type taken this wave per table
    std::map<uint32_t, bool> blocked;        // a table with a deferred request
    nkeys = 0;
    nops = 0;
    std::deque<request *> keep;
    const uint64_t cap_keys = s->cfg.max_wave_keys;
    const uint32_t cap_ops = s->cfg.max_wave_requests;
    for (request *r : s->pending) {
        // tables and slab sets are ordered separately (slab set ids in the upper half)
        const uint32_t key = r->slab >= 0 ? (0x80000000u | r->table) : r->table;
        bool ok = !blocked[key] && nops < cap_ops && nkeys + r->n <= cap_keys;
        auto it = table_op.find(key);
        if (ok && it != table_op.end() && conflicts(it->second, r->op)) ok = false;
        if (!ok) {
            blocked[key] = true;
            keep.push_back(r);
            continue;
        }
        table_op[key] = r->op;
        out.push_back(r);
        nkeys += r->n;
        nops++;
    }
    s->pending.swap(keep);
    (void)st;
    (void)ops_per_class;
    return out;
}

// One host copy into or out of the pinned staging buffers; src == nullptr
// zero-fills.
struct copy_job {
    void *dst;
    const void *src;
    uint64_t bytes;
};

// Copy one byte range [lo, hi) of the concatenated jobs.
void copy_range(const std::vector<copy_job> &jobs, uint64_t lo, uint64_t hi)
{
    uint64_t at = 0;
    for (const copy_job &j : jobs) {
        const uint64_t a = std::max(lo, at), b = std::min(hi, at + j.bytes);
        if (a < b) {
            char *d = static_cast<char *>(j.dst) + (a - at);
            if (j.src) memcpy(d, static_cast<const char *>(j.src) + (a - at), b - a);
            else memset(d, 0, b - a);
        }
        at += j.bytes;
        if (at >= hi) break;
    }
}

// Host threads that share a wave's copies into and out of pinned staging with
// the worker.  One thread's memcpy moves a fraction of what host memory and
// the PCIe link take (about 11 GB/s here), and waves under load hold tens of
// thousands of keys, so any copy of more than kCopyPart bytes is cut into
// equal parts of at least that size, taken by the worker and up to 8 pool
// threads (half the host's hardware threads at most).  The threads live as
// long as the server; a copy costs a wake-up, not a thread start.
struct copy_pool {
    static constexpr uint64_t kCopyPart = 128 << 10;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable go, finished;
    const std::vector<copy_job> *jobs = nullptr;
    uint64_t total = 0, gen = 0;
    unsigned nparts = 0, next = 0, done = 0;
    bool stop = false;

    void start()
    {
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned n = std::min(8u, hw / 2);
        for (unsigned k = 0; k < n; k++) {
            try {
                threads.emplace_back([this] { serve(); });
            } catch (const std::system_error &) {
                break;  // fewer helpers: the worker copies more itself
            }
        }
    }
    void shutdown()
    {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
        }
        go.notify_all();
        for (std::thread &t : threads) t.join();
        threads.clear();
    }
    ~copy_pool() { shutdown(); }
    // take parts of the current copy until none is left (lock held on entry and exit)
    void take_parts(std::unique_lock<std::mutex> &lk)
    {
        while (next < nparts) {
            const unsigned k = next++;
            const uint64_t lo = total * k / nparts, hi = total * (k + 1) / nparts;
            lk.unlock();
            copy_range(*jobs, lo, hi);
            lk.lock();
            if (++done == nparts) finished.notify_all();
        }
    }
    void serve()
    {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            go.wait(lk, [&] { return stop || gen != seen; });
            if (stop) return;
            seen = gen;
            take_parts(lk);
        }
    }
    // Run the copies of one wave; returns when every byte is copied.
    void run(const std::vector<copy_job> &js)
    {
        uint64_t t = 0;
        for (const copy_job &j : js) t += j.bytes;
        const uint64_t want = t / kCopyPart;
        const unsigned parts = (unsigned)std::min<uint64_t>(want, threads.size() + 1);
        if (parts <= 1) {
            copy_range(js, 0, t);
            return;
        }
        std::unique_lock<std::mutex> lk(mu);
        jobs = &js;
        total = t;
        nparts = parts;
        next = 0;
        done = 0;
        gen++;
        go.notify_all();
        take_parts(lk);
        finished.wait(lk, [&] { return done == nparts; });
        jobs = nullptr;
    }
};

// What a wave's copies and launches need from the server's tables, read
// while the lock is held: client threads may add tables meanwhile, which
// can move the table and class arrays.
struct wave_plan {
    std::vector<request *> reqs;
    std::vector<uint64_t> key_off;  // each request's first key in the staging buffers
    std::vector<uint32_t> vb;       // value bytes of its table
    std::vector<uint32_t> slot;     // its table's index in the class batch
    struct run {
        pg_batch *batch;
        cudaStream_t stream;
        uint32_t first, count, vb;
    };
    std::vector<run> runs;  // one pg_batch_run per kernel class, requests [first, first + count)
    struct slab_run {
        pg_slab_set *set;
        cudaStream_t stream;
        uint32_t req;
    };
    std::vector<slab_run> slab_runs;  // one bulk malloc / free per slab request
    uint64_t nkeys = 0;
    wave_layout lay{};
};

// Copy a finished wave's results out of the pinned staging buffers into the
// clients' buffers (without the lock: the requests belong to the worker until
// they are published).
void complete_stage(copy_pool &pool, pg_server::stage &st, const wave_plan &pl)
{
    std::vector<copy_job> jobs;
    for (size_t i = 0; i < pl.reqs.size(); i++) {
        request *r = pl.reqs[i];
        const uint64_t o = pl.key_off[i];
        const uint32_t vb = pl.vb[i];
        if (r->slab >= 0) {
            if (r->op == PG_OP_MALLOC && r->vals_out) jobs.push_back({r->vals_out, st.h + pl.lay.vout[0] + o * 8, r->n * 8});
            continue;
        }
        if (r->flags) jobs.push_back({r->flags, st.h + pl.lay.flags + o, r->n});
        if (r->op == PG_OP_QUERY && r->vals_out && vb)
            jobs.push_back({r->vals_out, st.h + pl.lay.vout[width_index(vb)] + o * vb, r->n * vb});
    }
    pool.run(jobs);
    const double t = now_s();
    const uint64_t *counts = reinterpret_cast<const uint64_t *>(st.h + pl.lay.counts);
    for (size_t i = 0; i < pl.reqs.size(); i++) {
        pl.reqs[i]->count = counts[i];
        pl.reqs[i]->t_done = t;
    }
}

void worker_loop(pg_server *s)
{
    cudaSetDevice(s->device);
    copy_pool pool;
    pool.start();
    struct slot_state {
        wave_plan plan;
        bool busy = false;
    } slots[kMaxWaves];
    int next_slot = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        // 1. complete finished waves (oldest first keeps per-table completion order)
        bool progressed = false;
        for (int k = 0; k < kMaxWaves; k++) {
            int w = (next_slot + k) % kMaxWaves;
            if (!slots[w].busy) continue;
            if (cudaEventQuery(s->stages[w].done) == cudaSuccess) {
                lk.unlock();
                const double c0 = now_s();
                complete_stage(pool, s->stages[w], slots[w].plan);
                const double c1 = now_s();
                lk.lock();
                s->t_copy_out += c1 - c0;
                for (request *r : slots[w].plan.reqs) {
                    if (r->slab >= 0) s->slabs[r->table].inflight--;
                    else s->tables[r->table].inflight--;
                    s->done[r->id] = r;
                }
                slots[w].plan = wave_plan();
                slots[w].busy = false;
                progressed = true;
            }
        }
        if (progressed) s->cv.notify_all();
        if (s->stop && s->pending.empty()) {
            bool any = false;
            for (auto &sl : slots) any |= sl.busy;
            if (!any) break;
        }
        // 2. launch a new wave into a free staging slot
        int w = -1;
        for (int k = 0; k < kMaxWaves; k++)
            if (!slots[(next_slot + k) % kMaxWaves].busy) {
                w = (next_slot + k) % kMaxWaves;
                break;
            }
        if (w >= 0 && !s->pending.empty()) {
            const double p0 = now_s();
            bool any_dirty = false;
            for (auto &k : s->classes) any_dirty |= k.dirty;
            if (any_dirty) {
                // a class's table list changed: let in-flight waves finish before its batch is rebuilt
                sync_all(s);
                for (auto &k : s->classes)
                    if (k.dirty) {
                        pg_status st = rebuild(s, k);
                        if (st != PG_OK) s->error = st;
                    }
            }
            pg_server::stage &st = s->stages[w];
            uint64_t nkeys;
            uint32_t nops;
            std::vector<uint32_t> opc;
            wave_plan &pl = slots[w].plan;
            pl.reqs = take_wave(s, st, nkeys, nops, opc);
            // group requests by class; each class's requests are contiguous in the op array
            // (slab requests after every table request)
            auto order = [&](const request *r) -> uint64_t {
                return r->slab >= 0 ? (1ull << 32) + r->table : (uint64_t)s->tables[r->table].cls;
            };
            std::stable_sort(pl.reqs.begin(), pl.reqs.end(),
                             [&](request *a, request *b) { return order(a) < order(b); });
            const size_t nr = pl.reqs.size();
            pl.key_off.assign(nr, 0);
            pl.vb.assign(nr, 0);
            pl.slot.assign(nr, 0);
            uint64_t ko = 0;
            for (size_t i = 0; i < nr; i++) {
                if (pl.reqs[i]->slab >= 0) {
                    slab_entry &se = s->slabs[pl.reqs[i]->table];
                    se.inflight++;
                    pl.key_off[i] = ko;
                    ko += pl.reqs[i]->n;
                    pl.slab_runs.push_back({se.set, se.stream, (uint32_t)i});
                    continue;
                }
                table_entry &te = s->tables[pl.reqs[i]->table];
                te.inflight++;
                pl.key_off[i] = ko;
                pl.vb[i] = s->classes[te.cls].vbytes;
                pl.slot[i] = te.slot;
                ko += pl.reqs[i]->n;
                if (i == 0 || te.cls != s->tables[pl.reqs[i - 1]->table].cls)
                    pl.runs.push_back({s->classes[te.cls].batch, s->classes[te.cls].stream, (uint32_t)i, 0,
                                       s->classes[te.cls].vbytes});
                pl.runs.back().count++;
            }
            pl.nkeys = ko;
            const double p1 = now_s();
            lk.unlock();
            // which value widths the wave moves, then its layout
            bool any_in[3] = {false, false, false}, any_q[3] = {false, false, false};
            for (size_t i = 0; i < nr; i++) {
                const request *r = pl.reqs[i];
                const uint32_t vb = pl.vb[i];
                if (r->slab >= 0) {
                    if (r->op == PG_OP_MALLOC) any_q[0] = true;  // the objects' addresses come back as 8-byte values
                } else if ((r->op == PG_OP_INSERT || r->op == PG_OP_INSERT_WITH_DELETE) && vb) {
                    any_in[width_index(vb)] = true;
                } else if (r->op == PG_OP_QUERY && vb) {
                    any_q[width_index(vb)] = true;
                }
            }
            pl.lay = lay_out(ko, nr, pl.runs.size(), any_in, any_q);
            const wave_layout &lay = pl.lay;
            // stage keys and values in pinned memory
            std::vector<copy_job> jobs;
            pg_op_desc *h_ops = reinterpret_cast<pg_op_desc *>(st.h + lay.ops);
            for (size_t i = 0; i < nr; i++) {
                request *r = pl.reqs[i];
                const uint64_t o = pl.key_off[i];
                const uint32_t vb = pl.vb[i];
                if (r->slab >= 0) {
                    // malloc: n sizes of 4 bytes; free: n pointers; both fit the keys' 8 bytes each
                    jobs.push_back({st.h + lay.keys + o * 8, r->keys, r->n * (r->op == PG_OP_MALLOC ? 4 : 8)});
                    h_ops[i] = pg_op_desc{0, r->op, o, r->n};
                    continue;
                }
                jobs.push_back({st.h + lay.keys + o * 8, r->keys, r->n * 8});
                if ((r->op == PG_OP_INSERT || r->op == PG_OP_INSERT_WITH_DELETE) && vb)
                    jobs.push_back({st.h + lay.vin[width_index(vb)] + o * vb, r->vals, r->n * vb});
                h_ops[i] = pg_op_desc{pl.slot[i], r->op, o, r->n};
            }
            pool.run(jobs);
            const double p2 = now_s();
            uint32_t *h_nops = reinterpret_cast<uint32_t *>(st.h + lay.nops);
            for (size_t ci = 0; ci < pl.runs.size(); ci++) h_nops[ci] = pl.runs[ci].count;
            memset(st.h + lay.counts, 0, nr * 8);
            // one copy in (upload stream), one run per class (its own stream,
            // after the upload), one copy out (download stream, after every run)
            cudaMemcpyAsync(st.d, st.h, lay.up_end, cudaMemcpyHostToDevice, s->stream);
            cudaEventRecord(st.uploaded, s->stream);
            unsigned char *d = st.d;
            uint64_t *d_keys = reinterpret_cast<uint64_t *>(d + lay.keys);
            pg_op_desc *d_ops = reinterpret_cast<pg_op_desc *>(d + lay.ops);
            uint32_t *d_nops = reinterpret_cast<uint32_t *>(d + lay.nops);
            uint64_t *d_counts = reinterpret_cast<uint64_t *>(d + lay.counts);
            uint8_t *d_flags = d + lay.flags;
            pg_status launch_error = PG_OK;
            for (size_t ci = 0; ci < pl.runs.size(); ci++) {
                const wave_plan::run &rn = pl.runs[ci];
                cudaStreamWaitEvent(rn.stream, st.uploaded, 0);
                const int x = width_index(rn.vb);
                pg_status rs = pg_batch_run(rn.batch, d_ops + rn.first, d_nops + ci, d_keys,
                                            lay.has_in[x] ? d + lay.vin[x] : nullptr,
                                            lay.has_out[x] ? d + lay.vout[x] : nullptr, d_flags, d_counts + rn.first,
                                            reinterpret_cast<pg_stream_t>(rn.stream));
                if (rs != PG_OK) launch_error = rs;
                // the download waits for this run (a wait takes the event's latest record)
                cudaEventRecord(st.ran, rn.stream);
                cudaStreamWaitEvent(s->down, st.ran, 0);
            }
            for (const wave_plan::slab_run &sr : pl.slab_runs) {
                const request *r = pl.reqs[sr.req];
                const uint64_t o = pl.key_off[sr.req];
                cudaStreamWaitEvent(sr.stream, st.uploaded, 0);
                pg_status rs;
                if (r->op == PG_OP_MALLOC)
                    rs = pg_slab_set_bulk_malloc(sr.set, reinterpret_cast<const uint32_t *>(d_keys + o), r->n,
                                                 reinterpret_cast<void **>(d + lay.vout[0] + o * 8), d_counts + sr.req,
                                                 reinterpret_cast<pg_stream_t>(sr.stream));
                else
                    rs = pg_slab_set_bulk_free(sr.set, reinterpret_cast<void *const *>(d_keys + o), r->n,
                                               d_counts + sr.req, reinterpret_cast<pg_stream_t>(sr.stream));
                if (rs != PG_OK) launch_error = rs;
                cudaEventRecord(st.ran, sr.stream);
                cudaStreamWaitEvent(s->down, st.ran, 0);
            }
            cudaMemcpyAsync(st.h + lay.counts, d + lay.counts, lay.end - lay.counts, cudaMemcpyDeviceToHost, s->down);
            cudaEventRecord(st.done, s->down);
            const double p3 = now_s();
            lk.lock();
            s->t_plan += p1 - p0;
            s->t_copy_in += p2 - p1;
            s->t_issue += p3 - p2;
            if (launch_error != PG_OK) s->error = launch_error;
            slots[w].busy = true;
            s->waves_run++;
            s->keys_run += ko;
            s->requests_run += nr;
            next_slot = (w + 1) % kMaxWaves;
            continue;
        }
        // 3. nothing to launch: wait for work or for a wave to finish
        bool any_busy = false;
        for (auto &sl : slots) any_busy |= sl.busy;
        const double w0 = now_s();
        if (any_busy) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
            lk.lock();
            s->t_wait_busy += now_s() - w0;
        } else {
            s->cv.wait_for(lk, std::chrono::milliseconds(2));
            s->t_wait_idle += now_s() - w0;
        }
    }
}

}  // namespace

extern "C" {

pg_status pg_server_create(const pg_server_config *cfg, pg_server **out)
{
    if (!cfg || !out || cfg->max_wave_keys == 0 || cfg->max_wave_requests == 0) return PG_ERR_INVALID;
    *out = nullptr;
    pg_server *s = new pg_server();
    s->cfg = *cfg;
    cudaGetDevice(&s->device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking);
    const uint64_t K = cfg->max_wave_keys, R = cfg->max_wave_requests;
    // the largest wave: every width in and out (one class run per request at most)
    const bool all[3] = {true, true, true};
    const uint64_t stage_bytes = lay_out(K, R, R, all, all).end;
    for (int w = 0; w < kMaxWaves && e == cudaSuccess; w++) {
        auto &st = s->stages[w];
        memset(&st, 0, sizeof(st));
        if (e == cudaSuccess) e = cudaMallocHost(&st.h, stage_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&st.d, stage_bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st.uploaded, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st.ran, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        pg_server_destroy(s);
        return e == cudaErrorMemoryAllocation ? PG_ERR_NOMEM : PG_ERR_CUDA;
    }
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return PG_OK;
}

pg_status pg_server_destroy(pg_server *s)
{
    if (!s) return PG_ERR_INVALID;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto &k : s->classes) {
        if (k.batch) pg_batch_destroy(k.batch);
        if (k.stream) cudaStreamDestroy(k.stream);
    }
    for (auto &te : s->tables)
        if (te.live) pg_table_destroy(te.t);
    for (auto &e : s->slabs) {
        if (e.set) pg_slab_set_destroy(e.set);
        if (e.stream) cudaStreamDestroy(e.stream);
    }
    for (auto &st : s->stages) {
        cudaFreeHost(st.h);
        cudaFree(st.d);
        if (st.uploaded) cudaEventDestroy(st.uploaded);
        if (st.ran) cudaEventDestroy(st.ran);
        if (st.done) cudaEventDestroy(st.done);
    }
    for (auto &kv : s->done) delete kv.second;
    for (request *r : s->pending) delete r;
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->down) cudaStreamDestroy(s->down);
    delete s;
    return PG_OK;
}

pg_status pg_server_add_table(pg_server *s, const pg_table_config *cfg, uint64_t seed, uint32_t *table_id)
{
    // the table is created on the current device, which must be the server's
    if (!s || !cfg || !table_id || !pg_on_device(s->device)) return PG_ERR_INVALID;
    // admission by HBM budget: the table's slot arrays (and fingerprints) must fit
    uint64_t need = 0;
    const uint32_t kb = cfg->format == PG_FMT_KV64 ? 8 : cfg->format == PG_FMT_PACKED_TAGVAL8 ? 1 : 2;
    const uint32_t vb = cfg->format == PG_FMT_KV64 ? 8
                        : (cfg->format == PG_FMT_TAGVAL16 || cfg->format == PG_FMT_PACKED_TAGVAL16) ? 2
                        : cfg->format == PG_FMT_PACKED_TAGVAL8                                       ? 1
                                                                                                     : 0;
    for (uint32_t l = 0; l < cfg->nlevels && l < 2; l++) {
        const pg_level_config &L = cfg->levels[l];
        if (L.bucket_size == 0 || L.nslots == 0) return PG_ERR_INVALID;
        const uint64_t nb = (L.nslots - 1) / L.bucket_size + 1;
        need += nb * L.bucket_size * (kb + vb);
        if (l == 0 && (cfg->flags & PG_TABLE_FINGERPRINTS)) need += nb * L.bucket_size;
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (s->bytes_used + need > s->cfg.hbm_budget_bytes) return PG_ERR_FULL;
    pg_table *t = nullptr;
    pg_status st = pg_table_create(cfg, seed, &t);
    if (st != PG_OK) return st;
    const uint32_t ck = class_key(t);
    uint32_t cls = (uint32_t)s->classes.size();
    for (uint32_t c = 0; c < s->classes.size(); c++) {
        const klass &k = s->classes[c];
        if (!k.tables.empty() && class_key(s->tables[k.tables[0]].t) == ck) {
            cls = c;
            break;
        }
    }
    if (cls == s->classes.size()) {
        cudaStream_t cs = nullptr;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            pg_table_destroy(t);
            return PG_ERR_CUDA;
        }
        s->classes.push_back(klass());
        s->classes.back().vbytes = vb;
        s->classes.back().stream = cs;
    }
    table_entry te;
    te.t = t;
    te.cls = cls;
    te.slot = (uint32_t)s->classes[cls].tables.size();
    te.bytes = pg_table_bytes(t);
    te.live = true;
    *table_id = (uint32_t)s->tables.size();
    s->tables.push_back(te);
    s->classes[cls].tables.push_back(*table_id);
    s->classes[cls].dirty = true;
    s->bytes_used += te.bytes;
    return PG_OK;
}

pg_status pg_server_drop_table(pg_server *s, uint32_t table_id)
{
    if (!s) return PG_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    if (table_id >= s->tables.size() || !s->tables[table_id].live) return PG_ERR_INVALID;
    for (request *r : s->pending)
        if (r->table == table_id) return PG_ERR_INVALID;  // collect its requests first
    if (s->tables[table_id].inflight) return PG_ERR_INVALID;  // and those already in a wave
    table_entry &te = s->tables[table_id];
    te.live = false;
    klass &k = s->classes[te.cls];
    k.tables.erase(std::remove(k.tables.begin(), k.tables.end(), table_id), k.tables.end());
    k.dirty = true;
    // waves already on the GPU may still use the table
    sync_all(s);
    pg_table_destroy(te.t);
    te.t = nullptr;
    s->bytes_used -= te.bytes;
    return PG_OK;
}

pg_table *pg_server_table(pg_server *s, uint32_t table_id)
{
    if (!s || table_id >= s->tables.size() || !s->tables[table_id].live) return nullptr;
    return s->tables[table_id].t;
}

uint64_t pg_server_bytes_in_use(pg_server *s)
{
    if (!s) return 0;
    std::lock_guard<std::mutex> g(s->mu);
    return s->bytes_used;
}

pg_status pg_server_submit(pg_server *s, uint32_t table_id, uint32_t op, const uint64_t *h_keys, const void *h_vals,
                           uint64_t n, void *h_vals_out, uint8_t *h_flags, uint64_t *request_id)
{
    if (!s || !request_id || (n && !h_keys) || op > PG_OP_INSERT_WITH_DELETE) return PG_ERR_INVALID;
    if (n > s->cfg.max_wave_keys) return PG_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    if (table_id >= s->tables.size() || !s->tables[table_id].live) return PG_ERR_INVALID;
    if (op == PG_OP_INSERT_WITH_DELETE && s->tables[table_id].t->ifmt != pg::FMT_PACKED16 &&
        s->tables[table_id].t->ifmt != pg::FMT_PACKED8)
        return PG_ERR_UNSUPPORTED;
    if (s->error != PG_OK) return s->error;
    request *r = new request();
    r->id = s->next_id++;
    r->table = table_id;
    r->slab = -1;
    r->op = op;
    r->keys = h_keys;
    r->vals = h_vals;
    r->n = n;
    r->vals_out = h_vals_out;
    r->flags = h_flags;
    r->count = 0;
    r->t_submit = now_s();
    r->t_done = 0;
    s->pending.push_back(r);
    s->outstanding.insert(r->id);
    *request_id = r->id;
    s->cv.notify_all();
    return PG_OK;
}

pg_status pg_server_add_slab_set(pg_server *s, uint32_t nclasses, const uint64_t *class_bytes,
                                 const uint64_t *num_allocs, uint32_t *set_id)
{
    if (!s || !class_bytes || !num_allocs || !set_id || nclasses == 0 || !pg_on_device(s->device))
        return PG_ERR_INVALID;
    // admission: every class's pool (whole slabs of 4096 objects) and its bitmaps
    uint64_t need = 0;
    for (uint32_t c = 0; c < nclasses; c++) {
        const uint64_t objs = (num_allocs[c] + 4095) / 4096 * 4096;
        need += objs * class_bytes[c] + objs / 8 + objs / 512;
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (s->bytes_used + need > s->cfg.hbm_budget_bytes) return PG_ERR_FULL;
    slab_entry e;
    pg_status st = pg_slab_set_create(nclasses, class_bytes, num_allocs, &e.set);
    if (st != PG_OK) return st;
    if (cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        pg_slab_set_destroy(e.set);
        return PG_ERR_CUDA;
    }
    e.bytes = need;
    e.live = true;
    *set_id = (uint32_t)s->slabs.size();
    s->slabs.push_back(e);
    s->bytes_used += need;
    return PG_OK;
}

pg_status pg_server_submit_slab(pg_server *s, uint32_t set_id, uint32_t op, const void *h_in, uint64_t n,
                                uint64_t *h_ptrs_out, uint64_t *request_id)
{
    if (!s || !request_id || (n && !h_in) || (op != PG_OP_MALLOC && op != PG_OP_FREE)) return PG_ERR_INVALID;
    if (n > s->cfg.max_wave_keys) return PG_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    if (set_id >= s->slabs.size() || !s->slabs[set_id].live) return PG_ERR_INVALID;
    if (s->error != PG_OK) return s->error;
    request *r = new request();
    r->id = s->next_id++;
    r->table = set_id;
    r->slab = (int32_t)set_id;
    r->op = op;
    r->keys = static_cast<const uint64_t *>(h_in);
    r->vals = nullptr;
    r->n = n;
    r->vals_out = h_ptrs_out;
    r->flags = nullptr;
    r->count = 0;
    r->t_submit = now_s();
    r->t_done = 0;
    s->pending.push_back(r);
    s->outstanding.insert(r->id);
    *request_id = r->id;
    s->cv.notify_all();
    return PG_OK;
}

pg_status pg_server_poll(pg_server *s, uint64_t request_id, int wait, uint64_t *count, double *latency_s)
{
    if (!s) return PG_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        auto it = s->done.find(request_id);
        if (it != s->done.end()) {
            request *r = it->second;
            if (count) *count = r->count;
            if (latency_s) *latency_s = r->t_done - r->t_submit;
            delete r;
            s->done.erase(it);
            s->outstanding.erase(request_id);
            return PG_OK;
        }
        // never issued, or already collected: nothing will complete it
        if (!s->outstanding.count(request_id)) return PG_ERR_INVALID;
        if (s->error != PG_OK) return s->error;
        if (!wait) return PG_ERR_TIMEOUT;  // not finished yet
        s->cv.wait_for(lk, std::chrono::milliseconds(1));
    }
}

pg_status pg_server_timing(pg_server *s, pg_server_timing_t *out)
{
    if (!s || !out) return PG_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    out->waves = s->waves_run;
    out->requests = s->requests_run;
    out->keys = s->keys_run;
    out->plan_s = s->t_plan;
    out->copy_in_s = s->t_copy_in;
    out->issue_s = s->t_issue;
    out->copy_out_s = s->t_copy_out;
    out->wait_busy_s = s->t_wait_busy;
    out->wait_idle_s = s->t_wait_idle;
    return PG_OK;
}

pg_status pg_server_stats(pg_server *s, uint64_t *waves, uint64_t *keys)
{
    if (!s) return PG_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    if (waves) *waves = s->waves_run;
    if (keys) *keys = s->keys_run;
    return PG_OK;
}

}  // extern "C"
