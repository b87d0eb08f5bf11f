// Serving loop of libadabool (abf_server_* in include/adabool.h): memory-
// budget admission, windowed continuous batching over a few CUDA streams,
// results resident in a device pool until released, and an open-loop trace
// replayer for latency measurements.
//
// The reference has no serving layer: its drivers answer one query per host
// call after an allocating, synchronous Prepare (test/adsfilter_q_all.cu:
// 412-440) or one batch of at most 32 (test/adsfilter_batch.cu:453-502).
//
// Threads: one server thread owns the streams, the workspaces and the
// launches; clients call submit / poll / release from any thread. All
// shared state (the waiting queue, the pool, the finished results) sits
// behind one mutex that is never held across a CUDA call.
#include "abf_kernels.cuh"
#include "abf_pool.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using abf::fail;

namespace {

uint64_t now_ns() {
    return uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(
                        std::chrono::steady_clock::now().time_since_epoch())
                        .count());
}

constexpr uint64_t kAlign = 256;
constexpr uint32_t kMaxStreams = 8;
uint64_t align_up(uint64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

struct Batch;

struct Req {
    uint64_t ticket = 0, tag = 0;
    std::vector<uint32_t> terms;
    uint64_t ids_bound = 0;  // min(n_ads, sum of list lengths)
    uint64_t t_arrival = 0;
    Batch* batch = nullptr;
    bool polled = false;
    abf_server_result res{};
};

struct Batch {
    std::vector<Req*> reqs;
    uint64_t off = 0;            // pool offset of the batch's range
    uint64_t bm_bytes = 0;       // bitmaps at [off, off + bm_bytes)
    uint64_t ids_bytes = 0;      // id room right after the bitmaps
    uint64_t ids_cap = 0;        // ids that fit the room
    bool bm_held = false, ids_held = false;
    uint32_t live = 0;           // queries not yet released
    abf_status status = ABF_OK;
    std::string error;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    abf_workspace* ws = nullptr;
    void* pinned = nullptr;
    uint32_t* h_terms = nullptr;
    uint64_t* h_off = nullptr;
    uint64_t* h_idoff = nullptr;
    uint8_t* h_paths = nullptr;
    uint32_t* h_err = nullptr;
    uint32_t* d_terms = nullptr;
    uint64_t* d_off = nullptr;
    uint64_t* d_idoff = nullptr;
    Batch* batch = nullptr;  // in flight
};

}  // namespace

struct abf_server {
    abf_index* ix = nullptr;
    abf_server_opts o{};
    uint64_t stride_words = 0;
    uint64_t bm_bytes = 0;  // one query's bitmap
    uint8_t* pool_base = nullptr;
    uint64_t pool_bytes = 0;
    abf::Pool pool;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> waiting;
    uint64_t waiting_terms = 0;
    std::deque<Req*> finished;                  // done, not yet polled
    std::unordered_map<uint64_t, Req*> held;    // done, not yet released
    uint64_t next_ticket = 1;
    bool stopping = false;
    bool blocked = false;  // head query waiting for pool room
    std::atomic<uint32_t> in_flight{0};  // batches launched and not finished
    abf_server_stats st{};
    std::thread th;
};

namespace {

bool want_ids(const abf_server* s) { return (s->o.outputs & ABF_SERVE_IDS) != 0; }
bool keep_bitmaps(const abf_server* s) { return (s->o.outputs & ABF_SERVE_BITMAPS) != 0; }

uint64_t room_of(const abf_server* s, uint64_t n, uint64_t ids) {
    return align_up(n * s->bm_bytes) + (want_ids(s) ? align_up(ids * 4) : 0);
}

void free_slot(Slot& sl) {
    if (sl.ws) abf_workspace_free(sl.ws);
    if (sl.pinned) cudaFreeHost(sl.pinned);
    if (sl.d_terms) cudaFree(sl.d_terms);
    if (sl.d_off) cudaFree(sl.d_off);
    if (sl.d_idoff) cudaFree(sl.d_idoff);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    sl = Slot{};
}

abf_status make_slot(abf_server* s, Slot& sl) {
    const uint32_t mq = s->o.max_batch_queries;
    const uint64_t mt = s->o.max_batch_terms;
    cudaError_t e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    const uint64_t pin = mt * 4 + (uint64_t(mq) + 1) * 16 + mq + 16;
    if (e == cudaSuccess) e = cudaMallocHost(&sl.pinned, pin);
    if (e == cudaSuccess) e = cudaMalloc(&sl.d_terms, std::max<uint64_t>(mt, 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sl.d_off, (uint64_t(mq) + 1) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sl.d_idoff, (uint64_t(mq) + 1) * 8);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? ABF_ERR_OOM : ABF_ERR_CUDA,
                    std::string("abf_server_create: ") + cudaGetErrorString(e));
    uint8_t* p = static_cast<uint8_t*>(sl.pinned);
    sl.h_off = reinterpret_cast<uint64_t*>(p);
    sl.h_idoff = sl.h_off + (mq + 1);
    sl.h_err = reinterpret_cast<uint32_t*>(sl.h_idoff + (mq + 1));
    sl.h_terms = sl.h_err + 4;
    sl.h_paths = reinterpret_cast<uint8_t*>(sl.h_terms + mt);
    return abf_workspace_create(s->ix, mq, std::max<uint64_t>(mt, 1), &sl.ws);
}

// Cuts a batch from the head of the waiting queue (caller holds s->mu).
Batch* cut_batch(abf_server* s) {
    const uint64_t largest = s->pool.largest();
    uint32_t n = 0;
    uint64_t terms = 0, ids = 0;
    bool short_of_room = false;
    for (Req* r : s->waiting) {
        if (n + 1 > s->o.max_batch_queries || terms + r->terms.size() > s->o.max_batch_terms) break;
        if (room_of(s, n + 1, ids + r->ids_bound) > largest) {
            short_of_room = true;
            break;
        }
        ++n;
        terms += r->terms.size();
        ids += r->ids_bound;
    }
    if (n == 0) {  // counted once per stretch of waiting at the head
        if (!s->blocked) ++s->st.admission_waits;
        s->blocked = true;
        return nullptr;
    }
    s->blocked = false;
    if (short_of_room) ++s->st.admission_waits;
    Batch* b = new Batch();
    b->bm_bytes = align_up(uint64_t(n) * s->bm_bytes);
    b->ids_cap = want_ids(s) ? ids : 0;
    b->ids_bytes = want_ids(s) ? align_up(ids * 4) : 0;
    b->off = s->pool.alloc(b->bm_bytes + b->ids_bytes);  // fits: <= largest extent
    b->bm_held = b->bm_bytes > 0;
    b->ids_held = b->ids_bytes > 0;
    b->reqs.reserve(n);
    for (uint32_t i = 0; i < n; ++i) {
        Req* r = s->waiting.front();
        s->waiting.pop_front();
        s->waiting_terms -= r->terms.size();
        r->batch = b;
        b->reqs.push_back(r);
    }
    b->live = n;
    s->st.reserved_bytes = s->pool.used();
    s->st.peak_reserved_bytes = std::max(s->st.peak_reserved_bytes, s->st.reserved_bytes);
    s->st.max_batch_queries_seen = std::max<uint64_t>(s->st.max_batch_queries_seen, n);
    return b;
}

// Enqueues one batch on a slot's stream: term upload, abf_batch_run, read
// back of id offsets / paths / error flag, completion event.
abf_status launch(abf_server* s, Slot& sl, Batch* b) {
    const uint32_t n = uint32_t(b->reqs.size());
    uint64_t nt = 0;
    sl.h_off[0] = 0;
    const uint64_t t = now_ns();
    for (uint32_t i = 0; i < n; ++i) {
        Req* r = b->reqs[i];
        if (!r->terms.empty()) std::memcpy(sl.h_terms + nt, r->terms.data(), r->terms.size() * 4);
        nt += r->terms.size();
        sl.h_off[i + 1] = nt;
        r->res.t_launch_ns = t;
    }
    cudaStream_t st = sl.stream;
    cudaError_t e = cudaSuccess;
    if (nt) e = cudaMemcpyAsync(sl.d_terms, sl.h_terms, nt * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.d_off, sl.h_off, (uint64_t(n) + 1) * 8, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(ABF_ERR_CUDA, std::string("server upload: ") + cudaGetErrorString(e));
    abf_batch bb{};
    bb.d_terms = sl.d_terms;
    bb.d_offsets = sl.d_off;
    bb.n_queries = n;
    bb.d_paths = nullptr;
    bb.path = s->o.path;
    bb.d_bitmaps = reinterpret_cast<uint32_t*>(s->pool_base + b->off);
    bb.bitmap_stride_words = s->stride_words;
    if (want_ids(s)) {
        bb.d_ids = reinterpret_cast<uint32_t*>(s->pool_base + b->off + b->bm_bytes);
        bb.ids_capacity = b->ids_cap;
        bb.d_id_offsets = sl.d_idoff;
    }
    abf_status rs = abf_batch_run(s->ix, sl.ws, &bb, st);
    if (rs != ABF_OK) return rs;
    if (want_ids(s)) e = cudaMemcpyAsync(sl.h_idoff, sl.d_idoff, (uint64_t(n) + 1) * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.h_paths, abf::ws_paths(sl.ws), n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.h_err, abf::ws_err(sl.ws), 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(sl.done, st);
    if (e != cudaSuccess) return fail(ABF_ERR_CUDA, std::string("server readback: ") + cudaGetErrorString(e));
    return ABF_OK;
}

// Fills the results of a batch whose event completed (or that failed) and
// hands them to pollers; trims the id room to the ids written.
void finish(abf_server* s, Slot* sl, Batch* b, abf_status status, const std::string& why) {
    const uint64_t t = now_ns();
    const uint32_t n = uint32_t(b->reqs.size());
    if (status == ABF_OK && sl && *sl->h_err) {
        status = (*sl->h_err & abf::kErrTermRange) ? ABF_ERR_CAPACITY : ABF_ERR_TIMEOUT;
        *sl->h_err = 0;
        cudaMemsetAsync(abf::ws_err(sl->ws), 0, 4, sl->stream);
    }
    if (status == ABF_OK && sl && want_ids(s) && sl->h_idoff[n] > b->ids_cap) status = ABF_ERR_CAPACITY;
    std::lock_guard<std::mutex> lk(s->mu);
    const uint32_t* bm0 = reinterpret_cast<const uint32_t*>(s->pool_base + b->off);
    const uint32_t* ids0 = reinterpret_cast<const uint32_t*>(s->pool_base + b->off + b->bm_bytes);
    for (uint32_t i = 0; i < n; ++i) {
        Req* r = b->reqs[i];
        abf_server_result& res = r->res;
        res.ticket = r->ticket;
        res.tag = r->tag;
        res.status = status;
        res.t_arrival_ns = r->t_arrival;
        res.t_done_ns = t;
        res.batch_queries = n;
        if (status == ABF_OK) {
            res.path = sl->h_paths[i];
            if (res.path < 5) ++s->st.path_queries[res.path];
            res.d_bitmap = keep_bitmaps(s) ? bm0 + uint64_t(i) * s->stride_words : nullptr;
            if (want_ids(s)) {
                res.d_ids = ids0 + sl->h_idoff[i];
                res.n_ids = sl->h_idoff[i + 1] - sl->h_idoff[i];
            }
        }
        s->finished.push_back(r);
        s->held[r->ticket] = r;
    }
    if (status == ABF_OK) {
        if (want_ids(s)) {  // trim the id room to what was written
            const uint64_t keep = align_up(sl->h_idoff[n] * 4);
            if (keep < b->ids_bytes) {
                s->pool.release(b->off + b->bm_bytes + keep, b->ids_bytes - keep);
                b->ids_bytes = keep;
                b->ids_held = keep > 0;
            }
        }
        if (!keep_bitmaps(s) && b->bm_held) {
            s->pool.release(b->off, b->bm_bytes);
            b->bm_held = false;
        }
    } else {
        ++s->st.failed_batches;
        b->error = why;
    }
    b->status = status;
    s->st.completed += n;
    ++s->st.batches;
    s->st.reserved_bytes = s->pool.used();
    s->cv_done.notify_all();
}

void release_batch(abf_server* s, Batch* b) {  // caller holds s->mu
    if (b->bm_held) s->pool.release(b->off, b->bm_bytes);
    if (b->ids_held) s->pool.release(b->off + b->bm_bytes, b->ids_bytes);
    for (Req* r : b->reqs) delete r;
    delete b;
    s->st.reserved_bytes = s->pool.used();
}

void server_loop(abf_server* s) {
    cudaSetDevice(s->ix->device);
    const uint64_t window = uint64_t(s->o.window_us) * 1000u;
    for (;;) {
        bool progressed = false;
        uint32_t in_flight = 0;
        for (Slot& sl : s->slots) {
            if (!sl.batch) continue;
            const cudaError_t e = cudaEventQuery(sl.done);
            if (e == cudaErrorNotReady) {
                ++in_flight;
                continue;
            }
            Batch* b = sl.batch;
            sl.batch = nullptr;
            s->in_flight.fetch_sub(1, std::memory_order_relaxed);
            finish(s, &sl, b, e == cudaSuccess ? ABF_OK : ABF_ERR_CUDA,
                   e == cudaSuccess ? std::string() : std::string(cudaGetErrorString(e)));
            progressed = true;
        }
        Slot* free_sl = nullptr;
        for (Slot& sl : s->slots)
            if (!sl.batch) {
                free_sl = &sl;
                break;
            }
        Batch* b = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stopping) {
                for (Req* r : s->waiting) {  // never launched: fail them
                    r->res.status = ABF_ERR_STATE;
                    delete r;
                }
                s->waiting.clear();
                s->waiting_terms = 0;
                if (in_flight == 0) break;
            } else if (free_sl && !s->waiting.empty()) {
                const uint64_t now = now_ns();
                const uint64_t oldest = s->waiting.front()->t_arrival;
                const bool cut = in_flight == 0 || s->waiting.size() >= s->o.max_batch_queries ||
                                 s->waiting_terms >= s->o.max_batch_terms || now >= oldest + window;
                if (cut) b = cut_batch(s);
            }
            if (!b && !progressed && in_flight == 0 && s->waiting.empty() && !s->stopping) {
                s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
                continue;
            }
        }
        if (b) {
            const abf_status rs = launch(s, *free_sl, b);
            if (rs == ABF_OK) {
                free_sl->batch = b;
                s->in_flight.fetch_add(1, std::memory_order_relaxed);
            } else {
                const std::string why = abf_last_error_string();
                cudaStreamSynchronize(free_sl->stream);  // nothing of it may still run
                finish(s, nullptr, b, rs, why);
            }
            progressed = true;
        }
        if (!progressed) std::this_thread::yield();
    }
}

void destroy_all(abf_server* s) {
    for (Slot& sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        free_slot(sl);
    }
    s->slots.clear();
    for (auto& kv : s->held) {
        Batch* b = kv.second->batch;
        if (b && --b->live == 0) {
            for (Req* r : b->reqs) delete r;
            delete b;
        }
    }
    s->held.clear();
    s->finished.clear();
    if (s->pool_base) cudaFree(s->pool_base);
    s->pool_base = nullptr;
}

}  // namespace

extern "C" {

uint64_t abf_clock_ns(void) { return now_ns(); }

abf_status abf_server_default_opts(abf_server_opts* o) {
    if (!o) return fail(ABF_ERR_INVALID, "null opts");
    *o = abf_server_opts{};
    o->budget_bytes = 40ull << 30;
    o->window_us = 100;
    o->max_batch_queries = 1024;
    o->max_batch_terms = 1ull << 22;
    o->n_streams = 4;
    o->path = ABF_PATH_AUTO;
    o->outputs = ABF_SERVE_BITMAPS | ABF_SERVE_IDS;
    return ABF_OK;
}

abf_status abf_server_create(abf_index* ix, const abf_server_opts* opts, abf_server** out) {
    try {
        if (!ix || !out) return fail(ABF_ERR_INVALID, "abf_server_create: null argument");
        *out = nullptr;
        if (!ix->on_device) return fail(ABF_ERR_STATE, "index has no device copy");
        abf_server_opts o{};
        if (opts) o = *opts;
        else abf_server_default_opts(&o);
        if (o.n_streams < 1 || o.n_streams > kMaxStreams) return fail(ABF_ERR_INVALID, "n_streams must be 1..8");
        if (o.max_batch_queries == 0 || o.max_batch_terms == 0)
            return fail(ABF_ERR_INVALID, "max_batch_queries and max_batch_terms must be positive");
        if (!(o.outputs & (ABF_SERVE_BITMAPS | ABF_SERVE_IDS)) || (o.outputs & ~(ABF_SERVE_BITMAPS | ABF_SERVE_IDS)))
            return fail(ABF_ERR_INVALID, "outputs must be a non-empty set of ABF_SERVE_BITMAPS / ABF_SERVE_IDS");
        if (uint32_t(o.path) > ABF_PATH_TILE) return fail(ABF_ERR_INVALID, "unknown path");
        if (ix->prof_on) return fail(ABF_ERR_STATE, "kernel timing is on for this index");
        std::unique_ptr<abf_server> s(new abf_server());
        s->ix = ix;
        s->o = o;
        s->stride_words = (uint64_t(ix->n_ads) + 127) / 128 * 4;
        s->bm_bytes = s->stride_words * 4;
        if (o.budget_bytes < s->bm_bytes) return fail(ABF_ERR_INVALID, "budget smaller than one bitmap");
        cudaError_t e = cudaSetDevice(ix->device);
        if (e != cudaSuccess) return fail(ABF_ERR_CUDA, cudaGetErrorString(e));
        s->pool_bytes = o.budget_bytes / kAlign * kAlign;
        e = cudaMalloc(&s->pool_base, s->pool_bytes);
        if (e != cudaSuccess) {
            s->pool_base = nullptr;
            return fail(ABF_ERR_OOM, std::string("server pool: ") + cudaGetErrorString(e));
        }
        s->pool.reset(s->pool_bytes);
        s->st.pool_bytes = s->pool_bytes;
        s->slots.resize(o.n_streams);
        for (Slot& sl : s->slots) {
            const abf_status st = make_slot(s.get(), sl);
            if (st != ABF_OK) {
                destroy_all(s.get());
                return st;
            }
        }
        s->th = std::thread(server_loop, s.get());
        *out = s.release();
        return ABF_OK;
    } catch (const std::bad_alloc&) {
        return fail(ABF_ERR_OOM, "host allocation failed");
    } catch (const std::exception& ex) {
        return fail(ABF_ERR_INTERNAL, ex.what());
    }
}

abf_status abf_server_submit(abf_server* s, const uint32_t* terms, uint32_t n_terms, uint64_t tag,
                             uint64_t arrival_ns, uint64_t* ticket) {
    try {
        if (!s || (n_terms && !terms)) return fail(ABF_ERR_INVALID, "abf_server_submit: bad arguments");
        if (n_terms > s->o.max_batch_terms) {
            std::lock_guard<std::mutex> lk(s->mu);
            ++s->st.rejected;
            return fail(ABF_ERR_CAPACITY, "query longer than max_batch_terms");
        }
        const abf_index* ix = s->ix;
        uint64_t sum = 0;
        for (uint32_t i = 0; i < n_terms; ++i)  // ids >= n_terms match nothing, as in abf_query
            if (terms[i] < ix->n_terms) sum += ix->h_term_len[terms[i]];
        std::unique_ptr<Req> r(new Req());
        r->terms.assign(terms, terms + n_terms);
        r->ids_bound = std::min<uint64_t>(sum, ix->n_ads);
        r->tag = tag;
        r->t_arrival = arrival_ns ? arrival_ns : now_ns();
        if (room_of(s, 1, r->ids_bound) > s->pool_bytes) {
            std::lock_guard<std::mutex> lk(s->mu);
            ++s->st.rejected;
            return fail(ABF_ERR_CAPACITY, "query's bitmap and id room exceed the pool");
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->stopping) return fail(ABF_ERR_STATE, "server is stopping");
            r->ticket = s->next_ticket++;
            if (ticket) *ticket = r->ticket;
            s->waiting_terms += n_terms;
            s->waiting.push_back(r.release());
            ++s->st.submitted;
        }
        s->cv_work.notify_one();
        return ABF_OK;
    } catch (const std::bad_alloc&) {
        return fail(ABF_ERR_OOM, "host allocation failed");
    }
}

abf_status abf_server_poll(abf_server* s, abf_server_result* out, uint32_t max_results, uint32_t timeout_us,
                           uint32_t* n_out) {
    if (!s || !n_out || (max_results && !out)) return fail(ABF_ERR_INVALID, "abf_server_poll: bad arguments");
    *n_out = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->finished.empty() && timeout_us)
        s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), [s] { return !s->finished.empty(); });
    uint32_t k = 0;
    while (k < max_results && !s->finished.empty()) {
        Req* r = s->finished.front();
        s->finished.pop_front();
        r->polled = true;
        out[k++] = r->res;
    }
    *n_out = k;
    return ABF_OK;
}

abf_status abf_server_release(abf_server* s, uint64_t ticket) {
    if (!s) return fail(ABF_ERR_INVALID, "null server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->held.find(ticket);
        if (it == s->held.end()) return fail(ABF_ERR_INVALID, "unknown or already released ticket");
        Req* r = it->second;
        if (!r->polled) return fail(ABF_ERR_STATE, "result not polled yet");
        s->held.erase(it);
        ++s->st.released;
        Batch* b = r->batch;
        if (--b->live == 0) release_batch(s, b);
    }
    s->cv_work.notify_one();
    return ABF_OK;
}

abf_status abf_server_get_stats(abf_server* s, abf_server_stats* out) {
    if (!s || !out) return fail(ABF_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->waiting = s->waiting.size();
    out->in_flight_batches = s->in_flight.load(std::memory_order_relaxed);
    out->reserved_bytes = s->pool.used();
    return ABF_OK;
}

abf_status abf_server_destroy(abf_server* s) {
    if (!s) return ABF_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    cudaSetDevice(s->ix->device);
    destroy_all(s);
    delete s;
    return ABF_OK;
}

abf_status abf_server_run_trace(abf_server* s, const uint32_t* terms, const uint64_t* offsets, uint32_t n,
                                const uint64_t* arrival_ns, double timeout_s, uint64_t* h_latency_ns,
                                uint64_t* h_queue_ns, uint64_t* h_n_ids, uint8_t* h_paths, abf_trace_stats* out) {
    try {
        if (!s || !offsets || !arrival_ns || !h_latency_ns || (offsets[n] && !terms))
            return fail(ABF_ERR_INVALID, "abf_server_run_trace: bad arguments");
        for (uint32_t i = 0; i < n; ++i) {
            h_latency_ns[i] = ~0ull;
            if (h_queue_ns) h_queue_ns[i] = ~0ull;
            if (h_n_ids) h_n_ids[i] = 0;
            if (h_paths) h_paths[i] = 0;
            if (i && arrival_ns[i] < arrival_ns[i - 1]) return fail(ABF_ERR_INVALID, "arrivals not ascending");
        }
        abf_trace_stats ts{};
        std::atomic<uint32_t> rejected{0};
        std::atomic<uint32_t> submitted{0};
        const uint64_t t0 = now_ns() + 2000000;  // 2 ms to start the generator
        std::thread gen([&] {
            for (uint32_t i = 0; i < n; ++i) {
                const uint64_t at = t0 + arrival_ns[i];
                while (now_ns() < at) {
                }
                const uint64_t len = offsets[i + 1] - offsets[i];
                if (abf_server_submit(s, terms + offsets[i], uint32_t(len), i, at, nullptr) != ABF_OK)
                    rejected.fetch_add(1, std::memory_order_relaxed);
                submitted.fetch_add(1, std::memory_order_release);
            }
        });
        const uint64_t deadline = t0 + (n ? arrival_ns[n - 1] : 0) + uint64_t(timeout_s * 1e9);
        std::vector<abf_server_result> buf(256);
        uint64_t seen = 0, last_done = t0;
        abf_status rc = ABF_OK;
        for (;;) {
            const uint32_t sub = submitted.load(std::memory_order_acquire);
            if (sub == n && seen + rejected.load() >= n) break;
            if (now_ns() > deadline) {
                rc = fail(ABF_ERR_TIMEOUT, "trace did not finish in time");
                break;
            }
            uint32_t k = 0;
            abf_server_poll(s, buf.data(), uint32_t(buf.size()), 1000, &k);
            for (uint32_t j = 0; j < k; ++j) {
                const abf_server_result& r = buf[j];
                const uint64_t i = r.tag;
                if (r.status == ABF_OK) {
                    h_latency_ns[i] = r.t_done_ns - r.t_arrival_ns;
                    if (h_queue_ns) h_queue_ns[i] = r.t_launch_ns - r.t_arrival_ns;
                    if (h_n_ids) h_n_ids[i] = r.n_ids;
                    if (h_paths) h_paths[i] = uint8_t(r.path);
                    ++ts.completed;
                } else {
                    ++ts.failed;
                }
                last_done = std::max(last_done, r.t_done_ns);
                abf_server_release(s, r.ticket);
            }
            seen += k;
        }
        gen.join();
        if (rc != ABF_OK) {  // drain what is still coming so the pool is clean
            for (int spins = 0; spins < 200; ++spins) {
                uint32_t k = 0;
                abf_server_poll(s, buf.data(), uint32_t(buf.size()), 5000, &k);
                for (uint32_t j = 0; j < k; ++j) abf_server_release(s, buf[j].ticket);
                abf_server_stats st{};
                abf_server_get_stats(s, &st);
                if (st.waiting == 0 && st.in_flight_batches == 0 && k == 0) break;
            }
        }
        ts.rejected = rejected.load();
        ts.seconds = double(last_done - (t0 + (n ? arrival_ns[0] : 0))) * 1e-9;
        if (out) *out = ts;
        return rc;
    } catch (const std::bad_alloc&) {
        return fail(ABF_ERR_OOM, "host allocation failed");
    } catch (const std::exception& ex) {
        return fail(ABF_ERR_INTERNAL, ex.what());
    }
}

}  // extern "C"
