// server.cu -- continuous-batching server over resident tables.
//
// No counterpart in the reference.  Clients submit requests {table, op, keys,
// values} from host memory at any time; a worker thread packs the pending
// requests into "waves" and keeps up to kMaxWaves waves on the GPU at once:
// while one wave runs, the next is staged and launched behind it, so requests
// that arrive while others are on the GPU join the next wave instead of
// waiting for the queue to drain.  A wave is one pinned staging copy in, one
// pg_batch_run per kernel class (tables of one format / bucket / scheme
// share a class), and one copy out, all on the server's stream.
//
// Ordering: requests on one table complete in submission order, and a wave
// never mixes conflicting requests on a table (only queries share a table
// with queries, inserts with inserts, removes with removes), so every result
// equals what the request returns when the requests are run one at a time in
// submission order (what the plain path does).
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
#include <thread>
#include <vector>

#include "poggers_b200.h"
#include "table_internal.h"

namespace {

constexpr int kMaxWaves = 2;

struct request {
    uint64_t id;
    uint32_t table;
    uint32_t op;
    const uint64_t *keys;
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
};

struct klass {
    pg_batch *batch = nullptr;
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
    cudaStream_t stream;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t bytes_used = 0;
    std::vector<table_entry> tables;
    std::vector<klass> classes;
    std::deque<request *> pending;
    std::map<uint64_t, request *> done;
    // staging (per wave slot): pinned host and device buffers
    struct stage {
        uint64_t *h_keys, *d_keys;
        // values by width (8, 2 and 1 bytes: uint64 tables, 16- and 8-bit
        // filters), each indexed like the keys; see width_index
        unsigned char *h_vin[3], *d_vin[3], *h_vout[3], *d_vout[3];
        uint8_t *h_flags, *d_flags;
        pg_op_desc *h_ops, *d_ops;
        uint32_t *h_nops, *d_nops;
        uint64_t *h_counts, *d_counts;
        cudaEvent_t done;
        bool busy;
    } stages[kMaxWaves];
    uint64_t waves_run = 0;
    uint64_t keys_run = 0;
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
        bool ok = !blocked[r->table] && nops < cap_ops && nkeys + r->n <= cap_keys;
        auto it = table_op.find(r->table);
        if (ok && it != table_op.end() && conflicts(it->second, r->op)) ok = false;
        if (!ok) {
            blocked[r->table] = true;
            keep.push_back(r);
            continue;
        }
        table_op[r->table] = r->op;
        out.push_back(r);
        nkeys += r->n;
        nops++;
    }
    s->pending.swap(keep);
    (void)st;
    (void)ops_per_class;
    return out;
}

void complete_stage(pg_server *s, pg_server::stage &st, std::vector<request *> &reqs, uint64_t *key_off)
{
    // copy results out of the pinned staging buffers into the clients' buffers
    uint32_t i = 0;
    for (request *r : reqs) {
        const uint64_t o = key_off[i];
        const table_entry &te = s->tables[r->table];
        const uint32_t vb = s->classes[te.cls].vbytes;
        if (r->flags) memcpy(r->flags, st.h_flags + o, r->n);
        if (r->op == PG_OP_QUERY && r->vals_out && vb)
            memcpy(r->vals_out, st.h_vout[width_index(vb)] + o * vb, r->n * vb);
        r->count = st.h_counts[i];
        r->t_done = now_s();
        i++;
    }
}

void worker_loop(pg_server *s)
{
    cudaSetDevice(s->device);
    struct slot_state {
        std::vector<request *> reqs;
        std::vector<uint64_t> key_off;
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
                complete_stage(s, s->stages[w], slots[w].reqs, slots[w].key_off.data());
                for (request *r : slots[w].reqs) s->done[r->id] = r;
                slots[w].reqs.clear();
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
            bool any_dirty = false;
            for (auto &k : s->classes) any_dirty |= k.dirty;
            if (any_dirty) {
                // a class's table list changed: let in-flight waves finish before its batch is rebuilt
                cudaStreamSynchronize(s->stream);
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
            std::vector<request *> reqs = take_wave(s, st, nkeys, nops, opc);
            // group requests by class; each class's requests are contiguous in the op array
            std::stable_sort(reqs.begin(), reqs.end(), [&](request *a, request *b) {
                return s->tables[a->table].cls < s->tables[b->table].cls;
            });
            slots[w].key_off.assign(reqs.size(), 0);
            uint64_t ko = 0;
            bool any_in[3] = {false, false, false}, any_q[3] = {false, false, false};
            for (size_t i = 0; i < reqs.size(); i++) {
                request *r = reqs[i];
                const table_entry &te = s->tables[r->table];
                const uint32_t vb = s->classes[te.cls].vbytes;
                slots[w].key_off[i] = ko;
                memcpy(st.h_keys + ko, r->keys, r->n * 8);
                if ((r->op == PG_OP_INSERT || r->op == PG_OP_INSERT_WITH_DELETE) && vb) {
                    unsigned char *dst = st.h_vin[width_index(vb)] + ko * vb;
                    if (r->vals) memcpy(dst, r->vals, r->n * vb);
                    else memset(dst, 0, r->n * vb);
                    any_in[width_index(vb)] = true;
                }
                if (r->op == PG_OP_QUERY && vb) any_q[width_index(vb)] = true;
                st.h_ops[i] = pg_op_desc{te.slot, r->op, ko, r->n};
                ko += r->n;
            }
            lk.unlock();
            // one copy in, one run per class, one copy out
            cudaMemcpyAsync(st.d_keys, st.h_keys, ko * 8, cudaMemcpyHostToDevice, s->stream);
            for (int x = 0; x < 3; x++)
                if (any_in[x])
                    cudaMemcpyAsync(st.d_vin[x], st.h_vin[x], ko * kWidths[x], cudaMemcpyHostToDevice, s->stream);
            cudaMemcpyAsync(st.d_ops, st.h_ops, reqs.size() * sizeof(pg_op_desc), cudaMemcpyHostToDevice, s->stream);
            cudaMemsetAsync(st.d_counts, 0, reqs.size() * 8, s->stream);
            size_t i = 0;
            uint32_t ci = 0;
            while (i < reqs.size()) {
                const uint32_t cls = s->tables[reqs[i]->table].cls;
                size_t j = i;
                while (j < reqs.size() && s->tables[reqs[j]->table].cls == cls) j++;
                st.h_nops[ci] = (uint32_t)(j - i);
                cudaMemcpyAsync(st.d_nops + ci, st.h_nops + ci, 4, cudaMemcpyHostToDevice, s->stream);
                const int x = width_index(s->classes[cls].vbytes);
                pg_status rs = pg_batch_run(s->classes[cls].batch, st.d_ops + i, st.d_nops + ci, st.d_keys,
                                            st.d_vin[x], st.d_vout[x], st.d_flags,
                                            st.d_counts + i, reinterpret_cast<pg_stream_t>(s->stream));
                if (rs != PG_OK) s->error = rs;
                i = j;
                ci++;
            }
            cudaMemcpyAsync(st.h_flags, st.d_flags, ko, cudaMemcpyDeviceToHost, s->stream);
            for (int x = 0; x < 3; x++)
                if (any_q[x])
                    cudaMemcpyAsync(st.h_vout[x], st.d_vout[x], ko * kWidths[x], cudaMemcpyDeviceToHost, s->stream);
            cudaMemcpyAsync(st.h_counts, st.d_counts, reqs.size() * 8, cudaMemcpyDeviceToHost, s->stream);
            cudaEventRecord(st.done, s->stream);
            lk.lock();
            slots[w].reqs = std::move(reqs);
            slots[w].busy = true;
            s->waves_run++;
            s->keys_run += ko;
            next_slot = (w + 1) % kMaxWaves;
            continue;
        }
        // 3. nothing to launch: wait for work or for a wave to finish
        bool any_busy = false;
        for (auto &sl : slots) any_busy |= sl.busy;
        if (any_busy) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
            lk.lock();
        } else {
            s->cv.wait_for(lk, std::chrono::milliseconds(2));
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
    const uint64_t K = cfg->max_wave_keys, R = cfg->max_wave_requests;
    for (int w = 0; w < kMaxWaves && e == cudaSuccess; w++) {
        auto &st = s->stages[w];
        memset(&st, 0, sizeof(st));
        if (e == cudaSuccess) e = cudaMallocHost(&st.h_keys, K * 8);
        if (e == cudaSuccess) e = cudaMalloc(&st.d_keys, K * 8);
        for (int x = 0; x < 3; x++) {
            if (e == cudaSuccess) e = cudaMallocHost(&st.h_vin[x], K * kWidths[x]);
            if (e == cudaSuccess) e = cudaMalloc(&st.d_vin[x], K * kWidths[x]);
            if (e == cudaSuccess) e = cudaMallocHost(&st.h_vout[x], K * kWidths[x]);
            if (e == cudaSuccess) e = cudaMalloc(&st.d_vout[x], K * kWidths[x]);
        }
        if (e == cudaSuccess) e = cudaMallocHost(&st.h_flags, K);
        if (e == cudaSuccess) e = cudaMalloc(&st.d_flags, K);
        if (e == cudaSuccess) e = cudaMallocHost(&st.h_ops, R * sizeof(pg_op_desc));
        if (e == cudaSuccess) e = cudaMalloc(&st.d_ops, R * sizeof(pg_op_desc));
        if (e == cudaSuccess) e = cudaMallocHost(&st.h_nops, 64 * 4);
        if (e == cudaSuccess) e = cudaMalloc(&st.d_nops, 64 * 4);
        if (e == cudaSuccess) e = cudaMallocHost(&st.h_counts, R * 8);
        if (e == cudaSuccess) e = cudaMalloc(&st.d_counts, R * 8);
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
    for (auto &k : s->classes)
        if (k.batch) pg_batch_destroy(k.batch);
    for (auto &te : s->tables)
        if (te.live) pg_table_destroy(te.t);
    for (auto &st : s->stages) {
        cudaFreeHost(st.h_keys);
        cudaFree(st.d_keys);
        for (int x = 0; x < 3; x++) {
            cudaFreeHost(st.h_vin[x]);
            cudaFree(st.d_vin[x]);
            cudaFreeHost(st.h_vout[x]);
            cudaFree(st.d_vout[x]);
        }
        cudaFreeHost(st.h_flags);
        cudaFree(st.d_flags);
        cudaFreeHost(st.h_ops);
        cudaFree(st.d_ops);
        cudaFreeHost(st.h_nops);
        cudaFree(st.d_nops);
        cudaFreeHost(st.h_counts);
        cudaFree(st.d_counts);
        if (st.done) cudaEventDestroy(st.done);
    }
    for (auto &kv : s->done) delete kv.second;
    for (request *r : s->pending) delete r;
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return PG_OK;
}

pg_status pg_server_add_table(pg_server *s, const pg_table_config *cfg, uint64_t seed, uint32_t *table_id)
{
    if (!s || !cfg || !table_id) return PG_ERR_INVALID;
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
        s->classes.push_back(klass());
        s->classes.back().vbytes = vb;
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
    table_entry &te = s->tables[table_id];
    te.live = false;
    klass &k = s->classes[te.cls];
    k.tables.erase(std::remove(k.tables.begin(), k.tables.end(), table_id), k.tables.end());
    k.dirty = true;
    // waves already on the GPU may still use the table
    cudaStreamSynchronize(s->stream);
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
            return PG_OK;
        }
        if (s->error != PG_OK) return s->error;
        if (!wait) return PG_ERR_TIMEOUT;  // not finished yet
        s->cv.wait_for(lk, std::chrono::milliseconds(1));
    }
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
