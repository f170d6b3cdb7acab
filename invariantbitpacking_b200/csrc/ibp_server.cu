// ibp_server.cu -- a continuous-batching decompress_fetch server.
//
// Clients submit requests (registered set, host row list, count) from any thread; a
// scheduler thread admits them in arrival order as output memory frees up, packs every
// admitted request into one batched launch (ibp_batch_fetch_hashed over the set registry:
// every (set, row) of the batch claimed in a hash table inside the fetch, so each crosses
// the bus once and its repeats are copied on the device; ibp_server_set_dedup picks the
// radix-sorted batch, ibp_batch_fetch_sorted, instead), and
// keeps up to `max_inflight` batches on the GPU at once, so requests that arrive while
// others run join the next launch instead of waiting for the queue to drain.  Completion is
// stamped by a thread that waits on each batch's event in launch order.
//
// Memory (all reserved at creation, nothing allocated per request):
//   * output arena: the caller's device buffer; a first-fit free list with coalescing hands
//     each request its rows, which stay valid until the client releases the request;
//   * index staging: a pinned host ring and a device ring of the same size; submit copies the
//     client's row list into the host ring, the batch copies its span to the device ring;
//   * request tables: one pinned + one device table per in-flight batch;
//   * one batch workspace (claim table or sort buffers) for max(index capacity, 2^20) rows
//     (batches run in stream order).
//
// The reference has no serving layer: its callers (ColossalAI embedding bags, FlexGen
// layers, DGL samplers) call decompress_fetch once per lookup.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ibp_internal.cuh"

namespace ibp200 {

using Clock = std::chrono::steady_clock;

static double now_us() {
    return std::chrono::duration<double, std::micro>(Clock::now().time_since_epoch()).count();
}

struct SrvRequest {
    int64_t id;
    int32_t set;
    int64_t count;
    int64_t first;
    bool has_index;
    int64_t idx_off;    // element offset of the row list in the index rings (-1: none)
    int64_t ring_end;   // ring position (monotonic) just past this request's row list
    int64_t out_off;    // byte offset in the output arena (-1: not admitted yet)
    int64_t out_bytes;
    double t_submit, t_admit, t_done;
    bool done = false;
    bool released = false;
};

struct Batch {
    std::vector<int64_t> ids;
    int64_t idx_begin = 0, idx_end = 0;  // index-ring span [begin, end), monotonic positions
    int table = 0;
    bool recorded = false;  // its completion event is in the stream
    bool complete = false;
};

struct Server {
    const void *registry = nullptr;
    std::vector<int64_t> set_v;      // words per row of each set
    std::vector<int64_t> set_n;
    int word_bytes = 8;
    int max_batch = 0, max_inflight = 2;
    char *arena = nullptr;
    size_t arena_bytes = 0;
    std::map<int64_t, int64_t> free_list;  // offset -> bytes
    int64_t *idx_host = nullptr, *idx_dev = nullptr;
    // ring positions are monotonic counters (physical slot = position % idx_cap):
    // [tail, head) is reserved, [tail, launched) already copied to the device
    int64_t idx_cap = 0, idx_head = 0, idx_tail = 0, idx_launched = 0;
    std::vector<char *> tbl_host, tbl_dev;
    std::vector<bool> tbl_busy;
    std::vector<cudaEvent_t> tbl_event;  // completion event of the batch using each table
    std::vector<cudaEvent_t> tbl_copied; // its index span and table are on the device
    void *ws = nullptr;
    size_t ws_bytes = 0;
    int64_t sort_cap = 0;  // rows a de-duplicating batch may hold (workspace size)
    int dedup = 0;         // 0: hashed batches, 1: sorted batches
    int64_t batch_rows = 0, batch_bytes = 0;  // admission limits of one batch
    cudaStream_t stream = nullptr;       // batch kernels, in launch order
    cudaStream_t copy_stream = nullptr;  // index spans and tables, ahead of their kernels
    int device = 0;

    std::mutex mu;
    std::condition_variable cv;       // scheduler wake-ups
    std::condition_variable done_cv;  // client waits
    std::condition_variable rec_cv;   // completion thread: a batch's event was recorded
    std::deque<int64_t> pending;
    int64_t pending_bytes = 0;  // output bytes of the queued (not yet admitted) requests
    std::map<int64_t, SrvRequest> reqs;
    std::deque<Batch *> inflight;
    int64_t next_id = 1;
    bool stop = false;
    std::thread thr, done_thr;
    std::string err;
    // stats
    int64_t batches = 0, rows_done = 0, bytes_done = 0;
};

static constexpr int kTableHeader = 64;
// Output bytes one batch admits by default (after its first request): ~2 ms of transfer at
// host-link speed, so a burst is served in arrival order by a pipeline of short launches
// instead of one launch that completes every request at its end.
static constexpr int64_t kDefaultBatchBytes = 128ll << 20;

// ---------------------------------------------------------------- arena allocation
static int64_t arena_alloc(Server *s, int64_t bytes) {
    bytes = (int64_t)align_up((size_t)bytes, 256);
    for (auto it = s->free_list.begin(); it != s->free_list.end(); ++it) {
        if (it->second >= bytes) {
            const int64_t off = it->first, left = it->second - bytes;
            s->free_list.erase(it);
            if (left > 0) s->free_list[off + bytes] = left;
            return off;
        }
    }
    return -1;
}

static void arena_free(Server *s, int64_t off, int64_t bytes) {
    bytes = (int64_t)align_up((size_t)bytes, 256);
    auto it = s->free_list.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != s->free_list.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        s->free_list.erase(nx);
    }
    if (it != s->free_list.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            s->free_list.erase(it);
        }
    }
}

// ---------------------------------------------------------------- index ring
static int64_t ring_used(const Server *s) { return s->idx_head - s->idx_tail; }

// Reserve n contiguous elements; a reservation never wraps (the ring skips to 0 instead).
static int64_t ring_reserve(Server *s, int64_t n) {
    if (n > s->idx_cap) return -1;
    int64_t pos = s->idx_head % s->idx_cap;
    int64_t skip = 0;
    if (pos + n > s->idx_cap) {
        skip = s->idx_cap - pos;
        pos = 0;
    }
    if (ring_used(s) + skip + n > s->idx_cap) return -1;
    s->idx_head += skip + n;
    return pos;
}

// ---------------------------------------------------------------- completion thread
// Waits for each batch's event in launch order and stamps its requests done.  An event
// rather than a host callback in the stream, so the next batch starts on the GPU without
// waiting for a host thread.
static void completer(Server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        Batch *b = nullptr;
        s->rec_cv.wait(lk, [&] {
            for (Batch *x : s->inflight)
                if (!x->complete) {
                    b = x->recorded ? x : nullptr;
                    return b != nullptr;
                }
            return s->stop;
        });
        if (!b) break;  // stopping and nothing left in flight
        const cudaEvent_t ev = s->tbl_event[b->table];
        lk.unlock();
        const cudaError_t e = cudaEventSynchronize(ev);
        const double t = now_us();
        lk.lock();
        if (e != cudaSuccess && s->err.empty()) s->err = cudaGetErrorString(e);
        for (int64_t id : b->ids) {
            auto it = s->reqs.find(id);
            if (it != s->reqs.end()) {
                it->second.t_done = t;
                it->second.done = true;
                s->rows_done += it->second.count;
                s->bytes_done += it->second.out_bytes;
            }
        }
        b->complete = true;
        s->cv.notify_all();
        s->done_cv.notify_all();
    }
}

// ---------------------------------------------------------------- scheduler
static void retire(Server *s) {
    // completed batches in launch order: free their index span and table
    while (!s->inflight.empty() && s->inflight.front()->complete) {
        Batch *b = s->inflight.front();
        s->inflight.pop_front();
        s->idx_tail = b->idx_end;
        s->tbl_busy[b->table] = false;
        delete b;
    }
}

static bool launch_batch_locked(Server *s, std::unique_lock<std::mutex> &lk) {
    int table = -1;
    for (int t = 0; t < (int)s->tbl_busy.size(); ++t)
        if (!s->tbl_busy[t]) {
            table = t;
            break;
        }
    if (table < 0 || s->pending.empty()) return false;
    Batch *b = new Batch();
    b->table = table;
    b->idx_begin = s->idx_launched;
    b->idx_end = s->idx_launched;
    std::vector<ibp_request> recs;
    int64_t rows = 0, out_bytes = 0;
    // a backlog (requests arriving faster than the link drains them) is split over the
    // launches that may be in flight, so batches grow with the queue: fewer, larger launches,
    // and rows that several queued requests of one set share cross the bus once
    const int64_t backlog_share = s->pending_bytes / std::max(1, s->max_inflight);
    const int64_t byte_limit = std::max(s->batch_bytes, backlog_share);
    // admit in arrival order while the output fits (head-of-line: an oversized request
    // waits for memory, later ones wait behind it to keep arrival order) and the rows fit
    // one de-duplicating batch
    while (!s->pending.empty() && (int)recs.size() < s->max_batch) {
        SrvRequest &r = s->reqs[s->pending.front()];
        if (!recs.empty() &&
            (rows + r.count > s->batch_rows || out_bytes + r.out_bytes > byte_limit))
            break;
        const int64_t off = arena_alloc(s, r.out_bytes);
        if (off < 0) break;
        r.out_off = off;
        r.t_admit = now_us();
        ibp_request q{};
        q.set = r.set;
        q.index = r.has_index ? s->idx_dev + r.idx_off : nullptr;
        q.first = r.first;
        q.count = r.count;
        q.out = s->arena + off;
        recs.push_back(q);
        rows += r.count;
        out_bytes += r.out_bytes;
        b->ids.push_back(r.id);
        b->idx_end = std::max(b->idx_end, r.ring_end);
        s->pending_bytes -= r.out_bytes;
        s->pending.pop_front();
    }
    if (recs.empty()) {
        delete b;
        return false;
    }
    s->idx_launched = b->idx_end;
    s->tbl_busy[table] = true;
    char *th = s->tbl_host[table], *td = s->tbl_dev[table];
    *reinterpret_cast<int32_t *>(th) = (int32_t)recs.size();
    std::memcpy(th + kTableHeader, recs.data(), sizeof(ibp_request) * recs.size());
    s->inflight.push_back(b);
    s->batches++;
    // the GPU work needs no lock: the rings and tables it touches are reserved
    lk.unlock();
    cudaSetDevice(s->device);
    // index span (one or two copies: the ring may have skipped to its start) and the request
    // table go on the copy stream, so they overlap the previous batch's kernel; the kernel
    // waits for them.  Ring spans and tables of batches in flight never overlap.
    const int64_t lo = b->idx_begin % s->idx_cap, n = b->idx_end - b->idx_begin;
    if (n > 0) {
        if (lo + n <= s->idx_cap) {
            cudaMemcpyAsync(s->idx_dev + lo, s->idx_host + lo, sizeof(int64_t) * n,
                            cudaMemcpyHostToDevice, s->copy_stream);
        } else {
            cudaMemcpyAsync(s->idx_dev + lo, s->idx_host + lo, sizeof(int64_t) * (s->idx_cap - lo),
                            cudaMemcpyHostToDevice, s->copy_stream);
            cudaMemcpyAsync(s->idx_dev, s->idx_host, sizeof(int64_t) * (n - (s->idx_cap - lo)),
                            cudaMemcpyHostToDevice, s->copy_stream);
        }
    }
    cudaMemcpyAsync(td, th, kTableHeader + sizeof(ibp_request) * recs.size(),
                    cudaMemcpyHostToDevice, s->copy_stream);
    cudaEventRecord(s->tbl_copied[table], s->copy_stream);
    cudaStreamWaitEvent(s->stream, s->tbl_copied[table], 0);
    // a batch that fits the workspace is de-duplicated (hash claims inside the fetch, or a
    // radix sort); a single range request beyond it (distinct rows in order) goes as listed
    const ibp_request *dreq = reinterpret_cast<const ibp_request *>(td + kTableHeader);
    ibp_status st;
    if (rows > s->sort_cap)
        st = ibp_batch_fetch(s->registry, dreq, reinterpret_cast<const int32_t *>(td),
                             s->max_batch, s->ws, s->ws_bytes, s->stream);
    else if (s->dedup == 1)
        st = ibp_batch_fetch_sorted(s->registry, dreq, (int32_t)recs.size(), rows, s->ws,
                                    s->ws_bytes, s->stream);
    else
        st = ibp_batch_fetch_hashed(s->registry, dreq, (int32_t)recs.size(), rows, s->ws,
                                    s->ws_bytes, s->stream);
    cudaEventRecord(s->tbl_event[table], s->stream);
    lk.lock();
    if (st != IBP_OK) s->err = ibp_last_error();
    b->recorded = true;
    s->rec_cv.notify_all();
    return true;
}

static void scheduler(Server *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        retire(s);
        bool launched = false;
        if ((int)s->inflight.size() < s->max_inflight && !s->pending.empty())
            launched = launch_batch_locked(s, lk);
        if (!launched) s->cv.wait_for(lk, std::chrono::milliseconds(5));
    }
}

// Frees every buffer, stream and event a server holds (null ones are skipped) and the server.
// Its threads must have stopped (or never started).
static void release_server(Server *s) {
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (char *h : s->tbl_host) cudaFreeHost(h);
    for (char *d : s->tbl_dev) cudaFree(d);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    for (cudaEvent_t ev : s->tbl_event) cudaEventDestroy(ev);
    for (cudaEvent_t ev : s->tbl_copied) cudaEventDestroy(ev);
    if (s->idx_host) cudaFreeHost(s->idx_host);
    if (s->idx_dev) cudaFree(s->idx_dev);
    if (s->ws) cudaFree(s->ws);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    for (Batch *b : s->inflight) delete b;
    delete s;
}

}  // namespace ibp200

using namespace ibp200;

extern "C" {

ibp_status ibp_server_create(const void *registry, const ibp_set_desc *sets, int32_t nsets,
                             int word_bytes, void *out_arena, size_t arena_bytes,
                             int64_t index_capacity, int32_t max_batch, int32_t max_inflight,
                             ibp_server **out) {
    clear_error();
    IBP_ARG(registry && sets && nsets > 0 && out_arena && out, "server_create: null argument");
    IBP_ARG(word_bytes == 4 || word_bytes == 8, "server_create: word size must be 4 or 8");
    IBP_ARG(max_batch > 0 && max_batch <= 8192, "server_create: max_batch must be 1..8192");
    IBP_ARG(max_inflight >= 1 && max_inflight <= 8, "server_create: max_inflight must be 1..8");
    IBP_ARG(index_capacity > 0, "server_create: index capacity must be positive");
    Server *s = new Server();
    s->registry = registry;
    for (int i = 0; i < nsets; ++i) {
        s->set_v.push_back(sets[i].vec_size);
        s->set_n.push_back(sets[i].num_vecs);
    }
    s->word_bytes = word_bytes;
    s->max_batch = max_batch;
    s->max_inflight = max_inflight;
    s->arena = (char *)out_arena;
    s->arena_bytes = arena_bytes;
    s->free_list[0] = (int64_t)(arena_bytes / 256 * 256);
    s->idx_cap = index_capacity;
    cudaGetDevice(&s->device);
    auto fail = [&](cudaError_t e, const char *what) {
        set_error("server_create: %s: %s", what, cudaGetErrorString(e));
        release_server(s);  // nothing of a failed creation is kept
        return IBP_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "copy stream");
    if ((e = cudaHostAlloc(&s->idx_host, sizeof(int64_t) * index_capacity, cudaHostAllocDefault)) != cudaSuccess) return fail(e, "index staging");
    if ((e = cudaMalloc(&s->idx_dev, sizeof(int64_t) * index_capacity)) != cudaSuccess) return fail(e, "device index ring");
    const size_t tbytes = kTableHeader + sizeof(ibp_request) * max_batch;
    for (int i = 0; i < max_inflight; ++i) {
        char *h = nullptr, *d = nullptr;
        if ((e = cudaHostAlloc(&h, tbytes, cudaHostAllocDefault)) != cudaSuccess) return fail(e, "table");
        s->tbl_host.push_back(h);
        if ((e = cudaMalloc(&d, tbytes)) != cudaSuccess) return fail(e, "table");
        s->tbl_dev.push_back(d);
        s->tbl_busy.push_back(false);
        cudaEvent_t ev = nullptr;
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
        s->tbl_event.push_back(ev);
        cudaEvent_t cev = nullptr;
        if ((e = cudaEventCreateWithFlags(&cev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
        s->tbl_copied.push_back(cev);
    }
    s->sort_cap = std::min<int64_t>(std::max<int64_t>(index_capacity, 1 << 20), INT32_MAX);
    s->batch_rows = s->sort_cap;
    s->batch_bytes = kDefaultBatchBytes;
    s->ws_bytes = std::max<size_t>(std::max(ibp_batch_fetch_sorted_workspace_size(s->sort_cap, max_batch),
                                            ibp_batch_fetch_hashed_workspace_size(s->sort_cap)),
                                   ibp_batch_fetch_workspace_size());
    if ((e = cudaMalloc(&s->ws, s->ws_bytes)) != cudaSuccess) return fail(e, "workspace");
    s->thr = std::thread(scheduler, s);
    s->done_thr = std::thread(completer, s);
    *out = reinterpret_cast<ibp_server *>(s);
    return IBP_OK;
}

// Queue a request: `count` rows of set `set`, either the listed rows (host array `rows`,
// copied before this returns) or, with rows == NULL, rows first .. first+count-1.  Returns
// its id in *id.  IBP_ERR_WORKSPACE when the index staging is full (retry later) or the
// request could never fit the output arena.
ibp_status ibp_server_submit(ibp_server *srv, int32_t set, const int64_t *rows, int64_t first,
                             int64_t count, int64_t *id) {
    clear_error();
    Server *s = reinterpret_cast<Server *>(srv);
    IBP_ARG(s && id, "server_submit: null argument");
    IBP_ARG(set >= 0 && set < (int32_t)s->set_v.size(), "server_submit: no set %d", set);
    IBP_ARG(count > 0, "server_submit: count must be positive");
    const int64_t out_bytes = count * s->set_v[set] * s->word_bytes;
    if ((size_t)out_bytes > s->arena_bytes) {
        set_error("server_submit: %lld output bytes exceed the %zu-byte arena", (long long)out_bytes,
                  s->arena_bytes);
        return IBP_ERR_WORKSPACE;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    SrvRequest r{};
    r.id = s->next_id++;
    r.set = set;
    r.count = count;
    r.first = first;
    r.has_index = rows != nullptr;
    r.idx_off = -1;
    r.out_off = -1;
    r.out_bytes = out_bytes;
    r.t_submit = now_us();
    if (rows) {
        retire(s);
        const int64_t pos = ring_reserve(s, count);
        if (pos < 0) {
            set_error("server_submit: index staging full (%lld of %lld entries in use)",
                      (long long)ring_used(s), (long long)s->idx_cap);
            return IBP_ERR_WORKSPACE;
        }
        std::memcpy(s->idx_host + pos, rows, sizeof(int64_t) * count);
        r.idx_off = pos;
    }
    r.ring_end = s->idx_head;
    s->reqs[r.id] = r;
    s->pending.push_back(r.id);
    s->pending_bytes += r.out_bytes;
    *id = r.id;
    lk.unlock();
    s->cv.notify_all();
    return IBP_OK;
}

// Wait (up to timeout_ms; < 0 forever) for request `id`; on success *out is its output rows
// (device memory, count x vec_size words) and times[0..2] = submit, admit, done (host
// microseconds, steady clock).  IBP_ERR_UNSUPPORTED on timeout.
ibp_status ibp_server_wait(ibp_server *srv, int64_t id, int32_t timeout_ms, void **out,
                           double *times) {
    clear_error();
    Server *s = reinterpret_cast<Server *>(srv);
    IBP_ARG(s, "server_wait: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] {
        auto it = s->reqs.find(id);
        return it == s->reqs.end() || it->second.done;
    };
    if (timeout_ms < 0)
        s->done_cv.wait(lk, ready);
    else if (!s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        set_error("server_wait: request %lld not done within %d ms", (long long)id, timeout_ms);
        return IBP_ERR_UNSUPPORTED;
    }
    auto it = s->reqs.find(id);
    IBP_ARG(it != s->reqs.end(), "server_wait: unknown request %lld", (long long)id);
    if (out) *out = s->arena + it->second.out_off;
    if (times) {
        times[0] = it->second.t_submit;
        times[1] = it->second.t_admit;
        times[2] = it->second.t_done;
    }
    if (!s->err.empty()) {
        set_error("server: %s", s->err.c_str());
        return IBP_ERR_CUDA;
    }
    return IBP_OK;
}

// Withdraw a request that is still queued (not yet admitted to a batch): it will not be
// fetched, and waiting for it afterwards reports an unknown request.  IBP_ERR_ARGUMENT for an
// unknown id; IBP_ERR_UNSUPPORTED once the request is admitted (wait for it and release it).
ibp_status ibp_server_cancel(ibp_server *srv, int64_t id) {
    clear_error();
    Server *s = reinterpret_cast<Server *>(srv);
    IBP_ARG(s, "server_cancel: null server");
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->reqs.find(id);
        IBP_ARG(it != s->reqs.end(), "server_cancel: unknown request %lld", (long long)id);
        if (it->second.out_off >= 0) {
            set_error("server_cancel: request %lld is already admitted", (long long)id);
            return IBP_ERR_UNSUPPORTED;
        }
        auto p = std::find(s->pending.begin(), s->pending.end(), id);
        if (p != s->pending.end()) {
            s->pending.erase(p);
            s->pending_bytes -= it->second.out_bytes;
        }
        s->reqs.erase(it);
    }
    s->cv.notify_all();
    s->done_cv.notify_all();
    return IBP_OK;
}

// Return a finished request's output rows to the arena.
ibp_status ibp_server_release(ibp_server *srv, int64_t id) {
    clear_error();
    Server *s = reinterpret_cast<Server *>(srv);
    IBP_ARG(s, "server_release: null server");
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->reqs.find(id);
        IBP_ARG(it != s->reqs.end() && it->second.done, "server_release: request %lld is not done",
                (long long)id);
        arena_free(s, it->second.out_off, it->second.out_bytes);
        s->reqs.erase(it);
    }
    s->cv.notify_all();
    return IBP_OK;
}

// Admission limits of one batch: at most max_rows rows (capped by the sort workspace) and
// max_bytes output bytes after its first request; <= 0 keeps the current value.
ibp_status ibp_server_set_batch_limits(ibp_server *srv, int64_t max_rows, int64_t max_bytes) {
    clear_error();
    Server *s = reinterpret_cast<Server *>(srv);
    IBP_ARG(s, "server_set_batch_limits: null server");
    std::lock_guard<std::mutex> g(s->mu);
    if (max_rows > 0) s->batch_rows = std::min(max_rows, s->sort_cap);
    if (max_bytes > 0) s->batch_bytes = max_bytes;
    return IBP_OK;
}

ibp_status ibp_server_set_dedup(ibp_server *srv, int32_t mode) {
    clear_error();
    Server *s = reinterpret_cast<Server *>(srv);
    IBP_ARG(s, "server_set_dedup: null server");
    IBP_ARG(mode == 0 || mode == 1, "server_set_dedup: mode must be 0 (hash) or 1 (sort)");
    std::lock_guard<std::mutex> g(s->mu);
    s->dedup = mode;
    return IBP_OK;
}

// stats[0..3] = batches launched, rows done, output bytes done, requests pending.
ibp_status ibp_server_stats(ibp_server *srv, int64_t *stats) {
    Server *s = reinterpret_cast<Server *>(srv);
    if (!s || !stats) return IBP_ERR_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    stats[0] = s->batches;
    stats[1] = s->rows_done;
    stats[2] = s->bytes_done;
    stats[3] = (int64_t)s->pending.size();
    return IBP_OK;
}

// Stop the scheduler after the in-flight batches finish and free the server's buffers.
ibp_status ibp_server_destroy(ibp_server *srv) {
    Server *s = reinterpret_cast<Server *>(srv);
    if (!s) return IBP_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->thr.joinable()) s->thr.join();
    s->rec_cv.notify_all();
    if (s->done_thr.joinable()) s->done_thr.join();
    release_server(s);
    return IBP_OK;
}

}  // extern "C"
