// C ABI of libadabool (include/adabool.h): index lifecycle, reference-shaped
// workers (prepare + run into a caller bitmap), the native batch runner and
// the single-query convenience call.
#include "abf_kernels.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <new>
#include <string>

namespace {
thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};
}  // namespace

namespace abf {
abf_status fail(abf_status s, const std::string& msg) {
    g_err = msg;
    return s;
}
void clear_error() { g_err.clear(); }
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace abf

using abf::fail;

#define CUDA_TRY(expr)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (expr);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return fail(e_ == cudaErrorMemoryAllocation ? ABF_ERR_OOM : ABF_ERR_CUDA,                    \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                             \
    } while (0)

#define ABF_TRY(expr)                      \
    do {                                   \
        abf_status s_ = (expr);            \
        if (s_ != ABF_OK) return s_;       \
    } while (0)

#define API_BEGIN try {
#define API_END                                                                 \
    }                                                                           \
    catch (const std::bad_alloc&) {                                             \
        return fail(ABF_ERR_OOM, "host allocation failed");                     \
    }                                                                           \
    catch (const std::exception& ex) {                                          \
        return fail(ABF_ERR_INTERNAL, ex.what());                               \
    }                                                                           \
    catch (...) {                                                               \
        return fail(ABF_ERR_INTERNAL, "unknown exception");                     \
    }

namespace {

// ---- kernel timing (abf_profile_enable / abf_profile_read) ----
enum Kid { K_PLAN, K_QUEUE, K_TILE, K_SCATTER, K_PROBE, K_COMPACT, K_PLANNER, K_GROUP, K_NKERNELS };
const char* const kKernelNames[K_NKERNELS] = {"plan",  "queue_scan", "tile_union", "scatter_union",
                                              "probe", "compact",    "planner",    "dense_group"};

struct Profiler {
    struct Rec {
        int kid;
        cudaEvent_t a, b;
    };
    std::vector<cudaEvent_t> pool;
    std::vector<Rec> recs;
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    ~Profiler() {
        for (auto& r : recs) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

// Records an event pair around one launch when timing is on.
struct ProfScope {
    abf_index* ix;
    int kid;
    cudaStream_t s;
    cudaEvent_t a = nullptr;
    ProfScope(abf_index* ix_, int kid_, cudaStream_t s_) : ix(ix_), kid(kid_), s(s_) {
        if (ix->prof_on && ix->prof) {
            a = static_cast<Profiler*>(ix->prof)->get();
            cudaEventRecord(a, s);
        }
    }
    ~ProfScope() {
        if (a) {
            auto* p = static_cast<Profiler*>(ix->prof);
            cudaEvent_t b = p->get();
            cudaEventRecord(b, s);
            p->recs.push_back({kid, a, b});
        }
    }
};

}  // namespace

#define TIMED(kid, expr)                \
    do {                                \
        ProfScope ps_(ix, (kid), s);    \
        CUDA_TRY(expr);                 \
    } while (0)

struct abf_workspace {
    abf_index* ix = nullptr;
    uint32_t max_q = 0;
    uint64_t max_terms = 0;
    uint32_t probe_cap = 0;
    uint64_t probe_stride = 0;
    uint32_t chunks_per_q = 0;
    uint32_t* heavy = nullptr;
    uint32_t* lpref = nullptr;
    uint32_t* tile_cls = nullptr;
    uint64_t* lcnt = nullptr;
    uint64_t* lpref_q = nullptr;
    uint32_t* probe_list = nullptr;
    uint32_t* n_probe = nullptr;
    uint32_t* probe_bm = nullptr;
    uint64_t* scan_status = nullptr;         // compaction look-back words, one per chunk (+1)
    unsigned long long* ticket = nullptr;   // compaction item counter
    uint64_t* id_off = nullptr;
    uint8_t* path_out = nullptr;
    uint8_t* auto_paths = nullptr;  // planner choices for ABF_PATH_AUTO batches
    uint16_t* q_dense16 = nullptr;  // the queries' dense bitmap lists (see PlanArgs)
    uint32_t* q_dstart = nullptr;   // per query
    uint32_t* q_ndense = nullptr;   // per query
    uint32_t* q_dmode = nullptr;    // per query
    uint32_t* err = nullptr;
    uint32_t* tile_list = nullptr;  // queries the merge kernel visits beside the dense group kernel
    uint32_t* n_tile_list = nullptr;
    uint32_t* sat = nullptr;        // per query: the dense group kernel's all-ones tiles, one bit each
    uint32_t sat_stride = 0;        // words per query (tiles of 32 words over n_ads)
    uint32_t* q_terms = nullptr;  // single-query staging (abf_query)
    uint64_t* q_off = nullptr;
    uint32_t spin_limit = abf::kDefaultSpinLimit;  // polls of every bounded device wait
};

struct abf_worker {
    abf_index* ix = nullptr;
    int kind = 0;  // 0 sparse, 1 dense (host bitmaps copied), 2 dense (caller device bitmaps)
    // sparse
    uint64_t n_keys = 0;
    uint32_t* d_keys = nullptr;
    uint64_t* d_off1 = nullptr;     // {0, n_keys}: the keys as one query
    uint64_t* d_offk = nullptr;     // 0..n_keys: every key its own query
    uint32_t* d_heavy = nullptr;
    uint32_t* d_lpref = nullptr;
    uint32_t* d_tile_cls = nullptr;
    uint64_t* d_lcnt = nullptr;
    uint64_t* d_lpref_q = nullptr;
    uint32_t* d_nprobe = nullptr;
    // dense
    uint64_t batch = 0;
    uint64_t len = 0;               // bytes per query bitmap as given
    uint32_t* d_qbm = nullptr;      // own copy, qbm_stride words per query
    uint64_t qbm_stride = 0;
    const uint8_t* d_ext = nullptr; // caller device bitmaps (kind 2)
};

namespace {

template <class T>
abf_status dev_alloc(T** p, uint64_t n, uint64_t* bytes = nullptr) {
    uint64_t b = std::max<uint64_t>(n, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), b);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(ABF_ERR_OOM, std::string("cudaMalloc(") + std::to_string(b) + "): " + cudaGetErrorString(e));
    }
    if (bytes) *bytes += b;
    return ABF_OK;
}

template <class T>
void dev_free(T*& p) {
    if (p) cudaFree(const_cast<void*>(reinterpret_cast<const void*>(p)));
    p = nullptr;
}

template <class T>
abf_status upload_vec(T** dst, const std::vector<T>& v, uint64_t* bytes) {
    ABF_TRY(dev_alloc(dst, v.size(), bytes));
    if (!v.empty()) CUDA_TRY(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return ABF_OK;
}

template <class T>
abf_status download_vec(std::vector<T>& v, const T* src, uint64_t n) {
    v.resize(n);
    if (n) CUDA_TRY(cudaMemcpy(v.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost));
    return ABF_OK;
}

uint64_t n_words_of(uint64_t n_bits) { return (n_bits + 31) / 32; }
uint64_t round4(uint64_t x) { return (x + 3) & ~uint64_t(3); }

void default_tuning(abf_index* ix) {
    abf_tuning& t = ix->tuning;
    t.tile_words = 2048;
    t.warps_per_tile = 8;
    // HYBRID merges per tile the lists that have dense bitmaps (at the
    // default dense_div, those holding at least 1/128 of the ads); measured on
    // the 2^24-ad workload, decoding shorter lists inside the tiles loses to
    // scattering them, as a tile holds only a block or two of each
    const uint32_t div = ix->dense_div && ix->dense_div != abf::kNone ? ix->dense_div : abf::kDefaultDenseDiv;
    t.heavy_min_len = uint32_t(std::max<uint64_t>((uint64_t(ix->n_ads) + div - 1) / div, abf::kBlock));
    t.probe_chunk_blocks = 256;
    t.scatter_blocks_per_warp = 8;
    t.ctas_per_sm = 6;
    t.probe_cap = 32;
    t.probe_min_fraction = 0.5f;
    t.group_min_queries = 32;
    t.fixed_tile_shape = 0;
    // the reference keeps a 256-id bucket as a bitset from 33 ids on
    // (src/AdaBool/inverted_list.h:425-458): a list of that density is
    // merged per tile by the fixed rule
    t.fixed_hybrid_min_len = uint32_t((33ull * ix->n_ads + 255) / 256);
    t.compact_ctas_per_sm = 6;
    t.group_tile_words = 0;
}

void free_device(abf_index* ix) {
    auto& d = ix->dev;
    dev_free(d.term_blk);
    dev_free(d.term_len);
    dev_free(d.blk_first);
    dev_free(d.blk_last);
    dev_free(d.blk_term);
    dev_free(d.blk_desc);
    dev_free(d.payload);
    dev_free(d.term_dense);
    dev_free(d.dense);
    dev_free(d.term_dir);
    dev_free(d.dir);
    dev_free(d.term_cbytes);
    dev_free(d.planner);
    d.bytes = 0;
    ix->on_device = false;
}

std::vector<uint32_t> cbytes32(const abf_index* ix) {
    std::vector<uint32_t> v(ix->h_term_bytes.size());
    for (size_t i = 0; i < v.size(); ++i) v[i] = uint32_t(std::min<uint64_t>(ix->h_term_bytes[i], 0xffffffffull));
    return v;
}

abf_status upload(abf_index* ix, int device) {
    CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    ix->sm_count = sms > 0 ? sms : 148;
    ix->device = device;
    auto& h = ix->host;
    auto& d = ix->dev;
    d.bytes = 0;
    abf_status st = ABF_OK;
    if ((st = upload_vec(&d.term_blk, h.term_blk, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.term_len, h.term_len, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.blk_first, h.blk_first, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.blk_last, h.blk_last, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.blk_term, h.blk_term, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.blk_desc, h.blk_desc, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.payload, h.payload, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.term_dense, ix->derived.term_dense, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.dense, ix->derived.dense, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.term_dir, ix->derived.term_dir, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.dir, ix->derived.dir, &d.bytes)) != ABF_OK ||
        (st = upload_vec(&d.term_cbytes, cbytes32(ix), &d.bytes)) != ABF_OK) {
        free_device(ix);
        return st;
    }
    ix->on_device = true;
    return ABF_OK;
}

abf_status finalize(abf_index* ix, const abf_build_opts* opts) {
    auto& h = ix->host;
    ix->n_terms = h.n_terms;
    ix->n_ads = h.n_ads;
    ix->n_postings = h.n_postings;
    ix->max_list_len = h.max_list_len;
    ix->n_blocks = h.n_blocks();
    ix->payload_units = h.payload.size();
    ix->h_term_blk = h.term_blk;
    ix->h_term_len = h.term_len;
    ix->h_term_bytes.assign(h.n_terms, 0);
    for (uint32_t t = 0; t < h.n_terms; ++t) {
        uint64_t bytes = 0;
        for (uint32_t b = h.term_blk[t]; b < h.term_blk[t + 1]; ++b) {
            const uint32_t meta = h.blk_desc[b].y;
            bytes += 16u + 16ull * abf::payload_units(abf::desc_count(meta), abf::desc_bits(meta));
        }
        ix->h_term_bytes[t] = bytes;
    }
    ix->host_valid = true;
    ix->dense_div = (opts && opts->dense_div) ? opts->dense_div : abf::kDefaultDenseDiv;
    abf::derive_tables(h, ix->dense_div, opts ? opts->n_threads : 0, &ix->derived);
    default_tuning(ix);
    uint32_t flags = opts ? opts->flags : 0u;
    if (!(flags & ABF_BUILD_HOST_ONLY)) {
        ABF_TRY(upload(ix, opts ? opts->device : 0));
        if (!(flags & ABF_BUILD_KEEP_HOST)) {
            ix->host = abf::HostIndex();
            ix->host_valid = false;
            // keep the small per-term tables, drop the bitmaps and directory
            ix->derived.dense = std::vector<uint32_t>();
            ix->derived.dir = std::vector<uint32_t>();
        }
    }
    return ABF_OK;
}

abf_status need_device(const abf_index* ix) {
    if (!ix) return fail(ABF_ERR_INVALID, "null index");
    if (!ix->on_device) return fail(ABF_ERR_STATE, "index has no device copy (built with ABF_BUILD_HOST_ONLY)");
    return ABF_OK;
}

void ws_release(abf_workspace* w) {
    dev_free(w->heavy);
    dev_free(w->lpref);
    dev_free(w->tile_cls);
    dev_free(w->lcnt);
    dev_free(w->lpref_q);
    dev_free(w->probe_list);
    dev_free(w->n_probe);
    dev_free(w->probe_bm);
    dev_free(w->scan_status);
    dev_free(w->ticket);
    dev_free(w->id_off);
    dev_free(w->path_out);
    dev_free(w->auto_paths);
    dev_free(w->q_dense16);
    dev_free(w->q_dstart);
    dev_free(w->q_ndense);
    dev_free(w->q_dmode);
    dev_free(w->err);
    dev_free(w->tile_list);
    dev_free(w->n_tile_list);
    dev_free(w->sat);
    dev_free(w->q_terms);
    dev_free(w->q_off);
}

abf_status ws_alloc(abf_index* ix, uint32_t max_q, uint64_t max_terms, uint64_t max_bits, abf_workspace* w) {
    w->ix = ix;
    w->max_q = max_q;
    w->max_terms = max_terms;
    w->probe_cap = ix->tuning.probe_cap;
    w->probe_stride = round4(n_words_of(ix->n_terms));
    w->chunks_per_q = abf::compact_chunks(std::max<uint64_t>(max_bits, ix->n_ads));
    const uint64_t chunks = uint64_t(max_q) * w->chunks_per_q;
    w->sat_stride = uint32_t((n_words_of(ix->n_ads) + 32u * 32u - 1u) / (32u * 32u));
    abf_status st;
    if ((st = dev_alloc(&w->heavy, max_q)) != ABF_OK || (st = dev_alloc(&w->lpref, max_terms)) != ABF_OK ||
        (st = dev_alloc(&w->tile_cls, max_terms)) != ABF_OK ||
        (st = dev_alloc(&w->lcnt, max_q)) != ABF_OK || (st = dev_alloc(&w->lpref_q, uint64_t(max_q) + 1)) != ABF_OK ||
        (st = dev_alloc(&w->probe_list, w->probe_cap)) != ABF_OK || (st = dev_alloc(&w->n_probe, 1)) != ABF_OK ||
        (st = dev_alloc(&w->probe_bm, uint64_t(w->probe_cap) * w->probe_stride)) != ABF_OK ||
        (st = dev_alloc(&w->scan_status, chunks + 1)) != ABF_OK || (st = dev_alloc(&w->ticket, 1)) != ABF_OK ||
        (st = dev_alloc(&w->id_off, uint64_t(max_q) + 1)) != ABF_OK ||
        (st = dev_alloc(&w->path_out, max_q)) != ABF_OK || (st = dev_alloc(&w->err, 1)) != ABF_OK ||
        (st = dev_alloc(&w->auto_paths, max_q)) != ABF_OK ||
        (st = dev_alloc(&w->q_dense16, max_terms + 8ull * max_q + 16)) != ABF_OK ||
        (st = dev_alloc(&w->q_dstart, max_q)) != ABF_OK || (st = dev_alloc(&w->q_ndense, max_q)) != ABF_OK ||
        (st = dev_alloc(&w->q_dmode, max_q)) != ABF_OK || (st = dev_alloc(&w->tile_list, max_q)) != ABF_OK ||
        (st = dev_alloc(&w->n_tile_list, 1)) != ABF_OK ||
        (st = dev_alloc(&w->sat, uint64_t(max_q) * w->sat_stride)) != ABF_OK ||
        (st = dev_alloc(&w->q_terms, max_terms)) != ABF_OK || (st = dev_alloc(&w->q_off, 2)) != ABF_OK) {
        ws_release(w);
        return st;
    }
    CUDA_TRY(cudaMemset(w->err, 0, sizeof(uint32_t)));
    return ABF_OK;
}

// the index's own workspace, grown to fit (growth synchronises the device)
abf_status own_ws(abf_index* ix, uint32_t n_q, uint64_t n_terms, uint64_t n_bits, abf_workspace** out) {
    abf_workspace* w = ix->own_ws;
    uint32_t need_chunks = abf::compact_chunks(std::max<uint64_t>(n_bits, ix->n_ads));
    if (w && w->max_q >= n_q && w->max_terms >= n_terms && w->chunks_per_q >= need_chunks &&
        w->probe_cap == ix->tuning.probe_cap) {
        *out = w;
        return ABF_OK;
    }
    uint32_t mq = std::max<uint32_t>(n_q, w ? w->max_q : 1u);
    uint64_t mt = std::max<uint64_t>({n_terms, w ? w->max_terms : 0ull, 4096ull});
    uint64_t mb = std::max<uint64_t>(n_bits, ix->n_ads);
    if (w) {
        CUDA_TRY(cudaDeviceSynchronize());
        ws_release(w);
    } else {
        w = new abf_workspace();
    }
    abf_status st = ws_alloc(ix, mq, mt, mb, w);
    if (st != ABF_OK) {
        delete w;
        ix->own_ws = nullptr;
        return st;
    }
    ix->own_ws = w;
    *out = w;
    return ABF_OK;
}

struct RunOpts {
    uint64_t* id_counts = nullptr;
};

abf_status run_compact(abf_index* ix, const abf::CompactArgs& ca, cudaStream_t s) {
    TIMED(K_COMPACT, abf::launch_compact(ca, ix->sm_count, ix->tuning.compact_ctas_per_sm, s));
    return ABF_OK;
}

abf_status run_batch(abf_index* ix, abf_workspace* ws, const abf_batch* b, const RunOpts& ro, cudaStream_t s) {
    if (b->n_queries == 0) return ABF_OK;
    if (b->n_queries > ws->max_q) return fail(ABF_ERR_CAPACITY, "batch has more queries than the workspace");
    const uint64_t n_words = n_words_of(ix->n_ads);
    if (b->bitmap_stride_words < n_words) return fail(ABF_ERR_INVALID, "bitmap_stride_words < (n_ads+31)/32");
    if (b->d_ids && !b->d_id_offsets && !ro.id_counts)
        return fail(ABF_ERR_INVALID, "d_ids needs d_id_offsets");
    CUDA_TRY(cudaSetDevice(ix->device));
    const abf::IndexView v = abf::view_of(ix);
    const abf_tuning& t = ix->tuning;
    CUDA_TRY(cudaMemsetAsync(ws->n_probe, 0, sizeof(uint32_t), s));
    CUDA_TRY(cudaMemsetAsync(ws->n_tile_list, 0, sizeof(uint32_t), s));
    abf::PlanArgs pa{};
    pa.terms = b->d_terms;
    pa.q_off = b->d_offsets;
    pa.n_q = b->n_queries;
    pa.paths = b->d_paths;
    pa.path_uniform = uint32_t(b->path);
    pa.hybrid_min = t.heavy_min_len;
    pa.probe_min_frac = t.probe_min_fraction;
    pa.fixed_hybrid_min = t.fixed_hybrid_min_len;
    pa.heavy_min = ws->heavy;
    pa.term_lpref = ws->lpref;
    pa.q_light_cnt = ws->lcnt;
    pa.probe_list = ws->probe_list;
    pa.n_probe = ws->n_probe;
    pa.probe_cap = ws->probe_cap;
    pa.path_out = ws->path_out;
    pa.max_terms = ws->max_terms;
    pa.err = ws->err;
    pa.dense_in_tile = 1;
    pa.tile_cls = ws->tile_cls;
    pa.q_dense16 = ws->q_dense16;
    pa.q_dstart = ws->q_dstart;
    pa.q_ndense = ws->q_ndense;
    pa.q_dmode = ws->q_dmode;
    pa.tile_list = ws->tile_list;
    pa.n_tile_list = ws->n_tile_list;
    // learned planner: the plan kernel runs its feature + MLP code for the
    // ABF_PATH_AUTO queries (no separate launch)
    pa.planner = ix->dev.planner;
    pa.n_postings = ix->n_postings;
    pa.probe_bm = ws->probe_bm;
    pa.probe_stride = ws->probe_stride;
    TIMED(K_PLAN, abf::launch_plan(v, pa, s));
    abf::QueueArgs qa{ws->lcnt, ws->lpref_q, b->n_queries};
    TIMED(K_QUEUE, abf::launch_queue_scan(qa, s));
    // the probe queries' term bitmaps are written by their plan CTAs
    const bool maybe_probe = ws->probe_cap > 0 && (b->d_paths || b->path == ABF_PATH_PROBE || b->path == ABF_PATH_AUTO);
    abf::TileArgs ta{};
    ta.tile_cls = ws->tile_cls;
    ta.q_off = b->d_offsets;
    ta.heavy_min = ws->heavy;
    ta.n_q = b->n_queries;
    // a batch too small to fill the GPU at the tuned tile shape (the tuner
    // sees large batches) gets full 8-warp CTAs first, then narrower tiles
    abf_tuning tt = t;
    if (!t.fixed_tile_shape) {
        const uint64_t want = 4ull * uint64_t(ix->sm_count) * 256u;  // threads
        auto threads = [&]() {
            return uint64_t(b->n_queries) * ((n_words + tt.tile_words - 1) / tt.tile_words) * tt.warps_per_tile * 32u;
        };
        while (tt.warps_per_tile < 8 && threads() < want) tt.warps_per_tile *= 2;
        while (tt.tile_words > 1024 && threads() < want) tt.tile_words >>= 1;
    }
    ta.n_tiles = uint32_t((n_words + tt.tile_words - 1) / tt.tile_words);
    ta.out = b->d_bitmaps;
    ta.out_stride = b->bitmap_stride_words;
    ta.n_words = n_words;
    ta.accumulate = 0;
    ta.vec_ok = (reinterpret_cast<uintptr_t>(b->d_bitmaps) % 16 == 0) && (b->bitmap_stride_words % 4 == 0);
    ta.q_dense16 = ws->q_dense16;
    ta.q_dstart = ws->q_dstart;
    ta.q_ndense = ws->q_ndense;
    ta.q_dmode = ws->q_dmode;
    ta.tile_list = ws->tile_list;
    ta.n_tile_list = ws->n_tile_list;
    // dense group kernel: the dense lists of every non-probe query in one pass per
    // tile, when the batch is large enough and the dense bitmaps (plus the
    // zero row) fit three TMA boxes of 256. Tiles of 64 words (two per lane:
    // half the index work per word) where two such stages and the batch's
    // lists (room for 64 per query) fit shared memory and the output rows
    // are 8-byte aligned, else 32 words.
    const uint32_t n_dense = v.n_dense;
    bool group = t.group_min_queries && b->n_queries >= t.group_min_queries && n_dense > 0 &&
                 n_dense + 1 <= abf::kGroupMaxBoxes * abf::kGroupBoxRows;
    const uint32_t wq = std::min<uint32_t>(b->n_queries, abf::kGroupMaxQueries);
    const bool out8 = reinterpret_cast<uintptr_t>(b->d_bitmaps) % 8 == 0 && b->bitmap_stride_words % 2 == 0;
    uint32_t gw = 32, stages = 2;
    if (out8 && abf::dense_group_list_cap(n_dense + 1, wq, 64, 2) >= 64u * wq) {
        gw = 64;
    } else if (out8 && abf::dense_group_list_cap(n_dense + 1, wq, 64, 1) > 0) {
        // one 64-word stage wherever it fits: the kernel keeps the window's
        // lists in shared memory beside it when they fit and reads them from
        // global memory otherwise; 32-word tiles cost twice the index work
        // per word (c1, 512-query windows: 5.60 against 7.46 ms per step)
        gw = 64;
        stages = 1;
    }
    if (t.group_tile_words == 32) {
        gw = 32;
        stages = abf::dense_group_list_cap(n_dense + 1, wq, 32, 2) > 0 ? 2u : 1u;
    }
    if (group && (ix->dense_tmap_base != ix->dev.dense || ix->dense_tmap_rows != n_dense ||
                  ix->dense_tmap_gw != gw)) {
        if (abf::encode_dense_tmap(v, gw, ix->dense_tmap) == cudaSuccess) {
            ix->dense_tmap_base = ix->dev.dense;
            ix->dense_tmap_rows = n_dense;
            ix->dense_tmap_gw = gw;
        } else {
            group = false;
        }
    }
    ta.skip_dense_only = group ? 1 : 0;
    // the group kernel marks each (query, tile) it leaves all ones; the
    // scatter then skips ORs into those tiles
    if (group) CUDA_TRY(cudaMemsetAsync(ws->sat, 0, uint64_t(b->n_queries) * ws->sat_stride * 4u, s));
    // one launch per window of at most kGroupMaxQueries queries (their
    // per-query state must fit the kernel's shared memory)
    for (uint32_t q0 = 0; group && q0 < b->n_queries; q0 += abf::kGroupMaxQueries) {
        abf::DenseGroupArgs ga{};
        ga.q_dense16 = ws->q_dense16;
        ga.q_dstart = ws->q_dstart + q0;
        ga.q_ndense = ws->q_ndense + q0;
        ga.q_dmode = ws->q_dmode + q0;
        ga.n_q = std::min<uint32_t>(abf::kGroupMaxQueries, b->n_queries - q0);
        ga.n_rows = n_dense + 1;
        ga.stages = stages;
        ga.list_cap = abf::dense_group_list_cap(ga.n_rows, ga.n_q, gw, stages);
        ga.n_tiles = uint32_t((n_words + gw - 1) / gw);
        ga.out = b->d_bitmaps + uint64_t(q0) * b->bitmap_stride_words;
        ga.out_stride = b->bitmap_stride_words;
        ga.n_words = n_words;
        ga.err = ws->err;
        ga.spin_limit = ws->spin_limit;
        ga.sat = ws->sat + uint64_t(q0) * ws->sat_stride;
        ga.sat_stride = ws->sat_stride;
        TIMED(K_GROUP, abf::launch_dense_group(ix->dense_tmap, gw, ga, ix->sm_count, s));
    }
    TIMED(K_TILE, abf::launch_tile_union(v, ta, tt, ix->sm_count, s));
    abf::ScatterArgs sa{};
    sa.terms = b->d_terms;
    sa.q_off = b->d_offsets;
    sa.term_lpref = ws->lpref;
    sa.q_light_pref = ws->lpref_q;
    sa.n_q = b->n_queries;
    sa.out = b->d_bitmaps;
    sa.out_stride = b->bitmap_stride_words;
    sa.blocks_per_warp = std::max<uint32_t>(1u, t.scatter_blocks_per_warp);
    if (group) {
        sa.sat = ws->sat;
        sa.sat_stride = ws->sat_stride;
        sa.sat_shift = gw == 64u ? 6u : 5u;
    }
    TIMED(K_SCATTER, abf::launch_scatter(v, sa, t, ix->sm_count, s));
    if (maybe_probe) {
        abf::ProbeArgs pr{};
        pr.qbm = ws->probe_bm;
        pr.qbm_stride = ws->probe_stride;
        pr.qbm_words = uint32_t(ws->probe_stride);
        pr.staged_ok = 1;
        pr.d_n_probe = ws->n_probe;
        pr.n_probe_host = ws->probe_cap;  // upper bound on the device count
        pr.out_slot = ws->probe_list;
        pr.out = b->d_bitmaps;
        pr.out_stride = b->bitmap_stride_words;
        pr.chunk_blocks = t.probe_chunk_blocks;
        pr.err = ws->err;
        pr.spin_limit = ws->spin_limit;
        TIMED(K_PROBE, abf::launch_probe(v, pr, t, ix->sm_count, s));
    }
    if (b->d_ids || ro.id_counts) {
        abf::CompactArgs ca{};
        ca.bm = b->d_bitmaps;
        ca.stride = b->bitmap_stride_words;
        ca.n_q = b->n_queries;
        ca.n_bits = ix->n_ads;
        ca.n_chunks = abf::compact_chunks(ix->n_ads);
        ca.status = ws->scan_status;
        ca.ticket = ws->ticket;
        ca.ids = b->d_ids;
        ca.capacity = b->d_ids ? b->ids_capacity : 0;
        ca.id_offsets = b->d_id_offsets ? b->d_id_offsets : ws->id_off;
        ca.id_counts = ro.id_counts;
        ca.err = ws->err;
        ca.spin_limit = ws->spin_limit;
        ABF_TRY(run_compact(ix, ca, s));
    }
    return ABF_OK;
}

abf_status worker_plan_scratch(abf_worker* w, uint64_t n_q) {
    ABF_TRY(dev_alloc(&w->d_heavy, n_q));
    ABF_TRY(dev_alloc(&w->d_lpref, std::max<uint64_t>(w->n_keys, 1)));
    ABF_TRY(dev_alloc(&w->d_tile_cls, std::max<uint64_t>(w->n_keys, 1)));
    ABF_TRY(dev_alloc(&w->d_lcnt, n_q));
    ABF_TRY(dev_alloc(&w->d_lpref_q, n_q + 1));
    ABF_TRY(dev_alloc(&w->d_nprobe, 1));
    return ABF_OK;
}

void worker_release(abf_worker* w) {
    dev_free(w->d_keys);
    dev_free(w->d_off1);
    dev_free(w->d_offk);
    dev_free(w->d_heavy);
    dev_free(w->d_lpref);
    dev_free(w->d_tile_cls);
    dev_free(w->d_lcnt);
    dev_free(w->d_lpref_q);
    dev_free(w->d_nprobe);
    dev_free(w->d_qbm);
}

// plan + scatter (and, for one query, merge tiles) of a sparse worker
abf_status run_sparse(const abf_worker* w, uint32_t* d_res, bool keyed, const uint32_t* d_qidx,
                      uint64_t res_stride_words, cudaStream_t s) {
    abf_index* ix = w->ix;
    ABF_TRY(need_device(ix));
    if (!d_res) return fail(ABF_ERR_INVALID, "null d_res");
    if (w->n_keys == 0) return ABF_OK;
    CUDA_TRY(cudaSetDevice(ix->device));
    const abf::IndexView v = abf::view_of(ix);
    const abf_tuning& t = ix->tuning;
    const uint32_t n_q = keyed ? uint32_t(w->n_keys) : 1u;
    const uint64_t* q_off = keyed ? w->d_offk : w->d_off1;
    abf::PlanArgs pa{};
    pa.terms = w->d_keys;
    pa.q_off = q_off;
    pa.n_q = n_q;
    // keyed batches may map several keys to one bitmap: only atomic
    // scatters are safe there; a single query merges its long lists per tile
    pa.path_uniform = keyed ? ABF_PATH_UNION : ABF_PATH_HYBRID;
    pa.hybrid_min = t.heavy_min_len;
    pa.heavy_min = w->d_heavy;
    pa.term_lpref = w->d_lpref;
    pa.q_light_cnt = w->d_lcnt;
    pa.n_probe = w->d_nprobe;
    pa.probe_cap = 0;
    pa.max_terms = w->n_keys;
    pa.err = nullptr;
    pa.dense_in_tile = keyed ? 0 : 1;
    pa.tile_cls = w->d_tile_cls;
    CUDA_TRY(cudaMemsetAsync(w->d_nprobe, 0, sizeof(uint32_t), s));
    TIMED(K_PLAN, abf::launch_plan(v, pa, s));
    abf::QueueArgs qa{w->d_lcnt, w->d_lpref_q, n_q};
    TIMED(K_QUEUE, abf::launch_queue_scan(qa, s));
    const uint64_t n_words = n_words_of(ix->n_ads);
    if (!keyed) {
        abf::TileArgs ta{};
        ta.tile_cls = w->d_tile_cls;
        ta.q_off = q_off;
        ta.heavy_min = w->d_heavy;
        ta.n_q = 1;
        ta.n_tiles = uint32_t((n_words + t.tile_words - 1) / t.tile_words);
        ta.out = d_res;
        ta.out_stride = n_words;
        ta.n_words = n_words;
        ta.accumulate = 1;
        ta.vec_ok = (reinterpret_cast<uintptr_t>(d_res) % 16 == 0) && (n_words % 4 == 0);
        TIMED(K_TILE, abf::launch_tile_union(v, ta, t, ix->sm_count, s));
    }
    abf::ScatterArgs sa{};
    sa.terms = w->d_keys;
    sa.q_off = q_off;
    sa.term_lpref = w->d_lpref;
    sa.q_light_pref = w->d_lpref_q;
    sa.n_q = n_q;
    sa.out_slot = keyed ? d_qidx : nullptr;
    sa.out = d_res;
    sa.out_stride = res_stride_words;
    sa.blocks_per_warp = std::max<uint32_t>(1u, t.scatter_blocks_per_warp);
    TIMED(K_SCATTER, abf::launch_scatter(v, sa, t, ix->sm_count, s));
    return ABF_OK;
}

abf_status run_dense(const abf_worker* w, uint32_t* d_res, uint64_t res_stride_words, cudaStream_t s) {
    abf_index* ix = w->ix;
    ABF_TRY(need_device(ix));
    if (!d_res) return fail(ABF_ERR_INVALID, "null d_res");
    if (w->batch == 0) return ABF_OK;
    CUDA_TRY(cudaSetDevice(ix->device));
    abf::ProbeArgs pr{};
    if (w->kind == 2) {
        pr.qbm = reinterpret_cast<const uint32_t*>(w->d_ext);
        pr.qbm_stride = w->len / 4;
        pr.qbm_words = uint32_t(std::min<uint64_t>(w->len / 4, 0xffffffffull));
        pr.staged_ok = (reinterpret_cast<uintptr_t>(w->d_ext) % 16 == 0) && ((w->len / 4) % 4 == 0);
    } else {
        pr.qbm = w->d_qbm;
        pr.qbm_stride = w->qbm_stride;
        pr.qbm_words = uint32_t(w->qbm_stride);
        pr.staged_ok = 1;
    }
    pr.d_n_probe = nullptr;
    pr.n_probe_host = uint32_t(w->batch);
    pr.out_slot = nullptr;
    pr.out = d_res;
    pr.out_stride = res_stride_words;
    pr.chunk_blocks = ix->tuning.probe_chunk_blocks;
    abf_workspace* ws = nullptr;
    ABF_TRY(own_ws(ix, 1, 1, ix->n_ads, &ws));
    pr.err = ws->err;
    pr.spin_limit = ws->spin_limit;
    TIMED(K_PROBE, abf::launch_probe(abf::view_of(ix), pr, ix->tuning, ix->sm_count, s));
    return ABF_OK;
}

}  // namespace

// ===========================================================================
// exported API
// ===========================================================================
extern "C" {

const char* abf_last_error_string(void) { return g_err.c_str(); }

const char* abf_status_string(abf_status s) {
    switch (s) {
        case ABF_OK: return "ok";
        case ABF_ERR_INVALID: return "invalid argument";
        case ABF_ERR_RANGE: return "id out of range";
        case ABF_ERR_CUDA: return "CUDA error";
        case ABF_ERR_OOM: return "out of memory";
        case ABF_ERR_STATE: return "invalid state";
        case ABF_ERR_IO: return "I/O error";
        case ABF_ERR_TIMEOUT: return "device wait timed out";
        case ABF_ERR_CAPACITY: return "capacity exceeded";
        default: return "internal error";
    }
}

uint32_t abf_abi_version(void) { return ABF_ABI_VERSION; }
uint64_t abf_launch_count(void) { return g_launches.load(); }

abf_status abf_index_build_csr(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms, uint32_t n_ads,
                               const abf_build_opts* opts, abf_index** out) {
    API_BEGIN
    abf::clear_error();
    if (!offsets || !out || n_terms == 0 || n_ads == 0) return fail(ABF_ERR_INVALID, "abf_index_build_csr: bad arguments");
    if (n_ads > (1u << 31)) return fail(ABF_ERR_RANGE, "n_ads above 2^31");
    if (n_terms > (1u << 31)) return fail(ABF_ERR_RANGE, "n_terms above 2^31");
    if (offsets[0] != 0) return fail(ABF_ERR_INVALID, "offsets[0] must be 0");
    for (uint32_t t = 0; t < n_terms; ++t)
        if (offsets[t + 1] < offsets[t]) return fail(ABF_ERR_INVALID, "offsets not monotone");
    if (offsets[n_terms] && !ads) return fail(ABF_ERR_INVALID, "null ads");
    *out = nullptr;
    abf_index* ix = new abf_index();
    abf_status st = abf::build_host(offsets, ads, n_terms, n_ads, opts ? opts->n_threads : 0, &ix->host);
    if (st == ABF_OK) st = finalize(ix, opts);
    if (st != ABF_OK) {
        free_device(ix);
        delete ix;
        return st;
    }
    *out = ix;
    return ABF_OK;
    API_END
}

abf_status abf_index_build_coo(const uint32_t* terms, const uint32_t* ads, uint64_t nnz, uint32_t n_terms,
                               uint32_t n_ads, const abf_build_opts* opts, abf_index** out) {
    API_BEGIN
    abf::clear_error();
    if (!out || n_terms == 0 || n_ads == 0 || (nnz && (!terms || !ads)))
        return fail(ABF_ERR_INVALID, "abf_index_build_coo: bad arguments");
    std::vector<uint64_t> off;
    std::vector<uint32_t> csr;
    ABF_TRY(abf::coo_to_csr(terms, ads, nnz, n_terms, n_ads, opts ? opts->n_threads : 0, &off, &csr));
    return abf_index_build_csr(off.data(), csr.data(), n_terms, n_ads, opts, out);
    API_END
}

abf_status abf_index_free(abf_index* ix) {
    API_BEGIN
    if (!ix) return ABF_OK;
    if (ix->on_device) {
        cudaSetDevice(ix->device);
        cudaDeviceSynchronize();
    }
    if (ix->own_ws) {
        ws_release(ix->own_ws);
        delete ix->own_ws;
    }
    if (ix->h_stage) cudaFreeHost(ix->h_stage);
    if (ix->stage_event) cudaEventDestroy(static_cast<cudaEvent_t>(ix->stage_event));
    delete static_cast<Profiler*>(ix->prof);
    ix->prof = nullptr;
    free_device(ix);
    delete ix;
    return ABF_OK;
    API_END
}

abf_status abf_index_get_stats(const abf_index* ix, abf_index_stats* o) {
    if (!ix || !o) return fail(ABF_ERR_INVALID, "null argument");
    o->n_terms = ix->n_terms;
    o->n_ads = ix->n_ads;
    o->n_postings = ix->n_postings;
    o->n_blocks = ix->n_blocks;
    o->payload_bytes = (ix->payload_units ? ix->payload_units - 1 : 0) * 16ull;
    o->device_bytes = ix->dev.bytes;
    o->max_list_len = ix->max_list_len;
    o->on_device = ix->on_device ? 1u : 0u;
    o->n_dense_lists = ix->derived.n_dense;
    o->n_directory_lists = ix->derived.n_dir;
    o->dense_bytes = uint64_t(ix->derived.n_dense) * ix->derived.dense_stride * 4u;
    return ABF_OK;
}

abf_status abf_index_list_lengths(const abf_index* ix, uint32_t* h_out, uint32_t n) {
    if (!ix || !h_out || n < ix->n_terms) return fail(ABF_ERR_INVALID, "abf_index_list_lengths: bad arguments");
    std::memcpy(h_out, ix->h_term_len.data(), size_t(ix->n_terms) * 4);
    return ABF_OK;
}

abf_status abf_index_decode_list(const abf_index* ix, uint32_t term, uint32_t* h_ids, uint64_t cap, uint64_t* n_out) {
    API_BEGIN
    if (!ix || !n_out) return fail(ABF_ERR_INVALID, "null argument");
    if (!ix->host_valid) return fail(ABF_ERR_STATE, "no host copy (build with ABF_BUILD_KEEP_HOST or HOST_ONLY)");
    if (term >= ix->n_terms) return fail(ABF_ERR_RANGE, "term >= n_terms");
    const auto& h = ix->host;
    *n_out = h.term_len[term];
    uint32_t buf[abf::kBlock];
    uint64_t k = 0;
    for (uint32_t b = h.term_blk[term]; b < h.term_blk[term + 1]; ++b) {
        abf::decode_block_host(h, b, buf);
        uint32_t cnt = abf::desc_count(h.blk_desc[b].y);
        for (uint32_t i = 0; i < cnt; ++i, ++k)
            if (h_ids && k < cap) h_ids[k] = buf[i];
    }
    return ABF_OK;
    API_END
}

}  // extern "C"

namespace {
// host copy of the list arrays from the device (for an index built without
// ABF_BUILD_KEEP_HOST)
abf_status fetch_host(const abf_index* ix, abf::HostIndex* h) {
    h->n_terms = ix->n_terms;
    h->n_ads = ix->n_ads;
    h->n_postings = ix->n_postings;
    h->max_list_len = ix->max_list_len;
    CUDA_TRY(cudaSetDevice(ix->device));
    ABF_TRY(download_vec(h->term_blk, ix->dev.term_blk, uint64_t(ix->n_terms) + 1));
    ABF_TRY(download_vec(h->term_len, ix->dev.term_len, ix->n_terms));
    ABF_TRY(download_vec(h->blk_first, ix->dev.blk_first, ix->n_blocks));
    ABF_TRY(download_vec(h->blk_last, ix->dev.blk_last, ix->n_blocks));
    ABF_TRY(download_vec(h->blk_term, ix->dev.blk_term, ix->n_blocks));
    ABF_TRY(download_vec(h->blk_desc, ix->dev.blk_desc, ix->n_blocks));
    ABF_TRY(download_vec(h->payload, ix->dev.payload, ix->payload_units));
    return ABF_OK;
}
}  // namespace

extern "C" {

abf_status abf_index_save(const abf_index* ix, const char* path) {
    API_BEGIN
    if (!ix || !path) return fail(ABF_ERR_INVALID, "null argument");
    if (ix->host_valid) return abf::save_host(ix->host, path);
    abf::HostIndex h;
    ABF_TRY(fetch_host(ix, &h));
    return abf::save_host(h, path);
    API_END
}

abf_status abf_index_set_dense_div(abf_index* ix, uint32_t dense_div) {
    API_BEGIN
    if (!ix) return fail(ABF_ERR_INVALID, "null index");
    abf::HostIndex tmp;
    const abf::HostIndex* h = &ix->host;
    if (!ix->host_valid) {
        ABF_TRY(fetch_host(ix, &tmp));
        h = &tmp;
    }
    abf::DerivedHost d;
    abf::derive_tables(*h, dense_div, 0, &d);
    if (ix->on_device) {
        CUDA_TRY(cudaSetDevice(ix->device));
        CUDA_TRY(cudaDeviceSynchronize());
        auto& dv = ix->dev;
        const uint64_t old = 4ull * (ix->derived.term_dense.size() + ix->derived.term_dir.size()) +
                             4ull * uint64_t(ix->derived.n_dense) * ix->derived.dense_stride +
                             4ull * uint64_t(ix->derived.n_dir) * ix->derived.dir_n;
        dev_free(dv.term_dense);
        dev_free(dv.dense);
        dev_free(dv.term_dir);
        dev_free(dv.dir);
        dv.bytes = dv.bytes > old ? dv.bytes - old : 0;
        abf_status st;
        if ((st = upload_vec(&dv.term_dense, d.term_dense, &dv.bytes)) != ABF_OK ||
            (st = upload_vec(&dv.dense, d.dense, &dv.bytes)) != ABF_OK ||
            (st = upload_vec(&dv.term_dir, d.term_dir, &dv.bytes)) != ABF_OK ||
            (st = upload_vec(&dv.dir, d.dir, &dv.bytes)) != ABF_OK) {
            free_device(ix);
            return st;
        }
        if (!ix->host_valid) {
            d.dense = std::vector<uint32_t>();
            d.dir = std::vector<uint32_t>();
        }
    }
    ix->derived = std::move(d);
    ix->dense_div = dense_div;
    return ABF_OK;
    API_END
}

abf_status abf_index_load(const char* path, const abf_build_opts* opts, abf_index** out) {
    API_BEGIN
    abf::clear_error();
    if (!path || !out) return fail(ABF_ERR_INVALID, "null argument");
    *out = nullptr;
    abf_index* ix = new abf_index();
    abf_status st = abf::load_host(path, &ix->host);
    if (st == ABF_OK) st = finalize(ix, opts);
    if (st != ABF_OK) {
        free_device(ix);
        delete ix;
        return st;
    }
    *out = ix;
    return ABF_OK;
    API_END
}

abf_status abf_index_to_device(abf_index* ix, int device) {
    API_BEGIN
    if (!ix) return fail(ABF_ERR_INVALID, "null index");
    if (ix->on_device) return ABF_OK;
    if (!ix->host_valid) return fail(ABF_ERR_STATE, "no host copy to upload");
    return upload(ix, device);
    API_END
}

abf_status abf_get_tuning(const abf_index* ix, abf_tuning* out) {
    if (!ix || !out) return fail(ABF_ERR_INVALID, "null argument");
    *out = ix->tuning;
    return ABF_OK;
}

abf_status abf_set_tuning(abf_index* ix, const abf_tuning* t) {
    if (!ix || !t) return fail(ABF_ERR_INVALID, "null argument");
    if (t->tile_words < 256 || t->tile_words > 16384 || (t->tile_words & (t->tile_words - 1)))
        return fail(ABF_ERR_INVALID, "tile_words must be a power of two from 256 to 16384");
    if (t->warps_per_tile != 1 && t->warps_per_tile != 2 && t->warps_per_tile != 4 && t->warps_per_tile != 8)
        return fail(ABF_ERR_INVALID, "warps_per_tile must be 1, 2, 4 or 8");
    if (t->probe_chunk_blocks == 0 || t->probe_chunk_blocks % 128 != 0)
        return fail(ABF_ERR_INVALID, "probe_chunk_blocks must be a positive multiple of 128");
    if (t->scatter_blocks_per_warp == 0 || t->ctas_per_sm == 0 || t->ctas_per_sm > 32)
        return fail(ABF_ERR_INVALID, "scatter_blocks_per_warp and ctas_per_sm (<= 32) must be positive");
    if (t->probe_cap > 65536) return fail(ABF_ERR_INVALID, "probe_cap above 65536");
    if (t->compact_ctas_per_sm == 0 || t->compact_ctas_per_sm > 6)
        return fail(ABF_ERR_INVALID, "compact_ctas_per_sm must be 1..6");
    if (t->group_tile_words != 0 && t->group_tile_words != 32 && t->group_tile_words != 64)
        return fail(ABF_ERR_INVALID, "group_tile_words must be 0, 32 or 64");
    ix->tuning = *t;
    return ABF_OK;
}

// ---------------------------------------------------------------------------
// reference-shaped workers
// ---------------------------------------------------------------------------
abf_status abf_prepare_sparse(abf_index* ix, const uint32_t* keys, uint64_t n_keys, abf_worker** out) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!out || (n_keys && !keys)) return fail(ABF_ERR_INVALID, "abf_prepare_sparse: bad arguments");
    if (n_keys >= (1ull << 32)) return fail(ABF_ERR_RANGE, "too many keys");
    CUDA_TRY(cudaSetDevice(ix->device));
    *out = nullptr;
    abf_worker* w = new abf_worker();
    w->ix = ix;
    w->kind = 0;
    w->n_keys = n_keys;
    std::vector<uint64_t> offk(n_keys + 1);
    for (uint64_t i = 0; i <= n_keys; ++i) offk[i] = i;
    uint64_t off1[2] = {0, n_keys};
    abf_status st = ABF_OK;
    if ((st = dev_alloc(&w->d_keys, n_keys)) != ABF_OK || (st = dev_alloc(&w->d_off1, 2)) != ABF_OK ||
        (st = dev_alloc(&w->d_offk, n_keys + 1)) != ABF_OK ||
        (st = worker_plan_scratch(w, std::max<uint64_t>(n_keys, 1))) != ABF_OK) {
        worker_release(w);
        delete w;
        return st;
    }
    cudaError_t e = cudaSuccess;
    if (n_keys) e = cudaMemcpy(w->d_keys, keys, n_keys * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(w->d_off1, off1, sizeof(off1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(w->d_offk, offk.data(), offk.size() * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        worker_release(w);
        delete w;
        return fail(ABF_ERR_CUDA, std::string("abf_prepare_sparse upload: ") + cudaGetErrorString(e));
    }
    *out = w;
    return ABF_OK;
    API_END
}

static abf_status prepare_dense_impl(abf_index* ix, uint64_t batch, uint64_t len, const uint8_t* bm, bool device,
                                     abf_worker** out) {
    ABF_TRY(need_device(ix));
    if (!out || (batch && !bm)) return fail(ABF_ERR_INVALID, "dense prepare: bad arguments");
    if (batch > 1 && len % 4 != 0) return fail(ABF_ERR_INVALID, "batch bitmap length must be a multiple of 4 bytes");
    CUDA_TRY(cudaSetDevice(ix->device));
    *out = nullptr;
    abf_worker* w = new abf_worker();
    w->ix = ix;
    w->batch = batch;
    w->len = len;
    if (device) {
        w->kind = 2;
        w->d_ext = bm;
        *out = w;
        return ABF_OK;
    }
    w->kind = 1;
    // own copy, padded so every query covers all n_terms bits and starts
    // 16-byte aligned (bulk copies into shared memory need both)
    w->qbm_stride = round4(std::max<uint64_t>(n_words_of(ix->n_terms), 1));
    abf_status st = dev_alloc(&w->d_qbm, std::max<uint64_t>(batch, 1) * w->qbm_stride);
    if (st != ABF_OK) {
        delete w;
        return st;
    }
    const uint64_t copy = std::min<uint64_t>(len, w->qbm_stride * 4);
    cudaError_t e = cudaMemset(w->d_qbm, 0, std::max<uint64_t>(batch, 1) * w->qbm_stride * 4);
    if (e == cudaSuccess && batch && copy)
        e = cudaMemcpy2D(w->d_qbm, w->qbm_stride * 4, bm, len, copy, batch, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        worker_release(w);
        delete w;
        return fail(ABF_ERR_CUDA, std::string("dense prepare upload: ") + cudaGetErrorString(e));
    }
    *out = w;
    return ABF_OK;
}

abf_status abf_prepare_dense(abf_index* ix, uint64_t len, const uint8_t* bm, abf_worker** out) {
    API_BEGIN
    return prepare_dense_impl(ix, 1, len, bm, false, out);
    API_END
}

abf_status abf_prepare_batch(abf_index* ix, uint64_t batch, uint64_t len, const uint8_t* bm, abf_worker** out) {
    API_BEGIN
    return prepare_dense_impl(ix, batch, len, bm, false, out);
    API_END
}

abf_status abf_prepare_batch_device(abf_index* ix, uint64_t batch, uint64_t len, const uint8_t* d_bm,
                                    abf_worker** out) {
    API_BEGIN
    return prepare_dense_impl(ix, batch, len, d_bm, true, out);
    API_END
}

abf_status abf_worker_free(abf_worker* w) {
    API_BEGIN
    if (!w) return ABF_OK;
    if (w->ix && w->ix->on_device) {
        cudaSetDevice(w->ix->device);
        cudaDeviceSynchronize();
    }
    worker_release(w);
    delete w;
    return ABF_OK;
    API_END
}

abf_status abf_list_union_sparse(const abf_worker* w, uint32_t* d_res, void* stream) {
    API_BEGIN
    if (!w || w->kind != 0) return fail(ABF_ERR_INVALID, "abf_list_union_sparse needs a sparse worker");
    return run_sparse(w, d_res, false, nullptr, n_words_of(w->ix->n_ads), static_cast<cudaStream_t>(stream));
    API_END
}

abf_status abf_batch_list_union_sparse(const abf_worker* w, uint32_t* d_res, const uint32_t* d_qidx,
                                       uint32_t res_len_bytes, void* stream) {
    API_BEGIN
    if (!w || w->kind != 0) return fail(ABF_ERR_INVALID, "abf_batch_list_union_sparse needs a sparse worker");
    if (!d_qidx && w->n_keys) return fail(ABF_ERR_INVALID, "null d_qidx");
    if (uint64_t(res_len_bytes) * 8 < w->ix->n_ads) return fail(ABF_ERR_INVALID, "res_len_bytes smaller than the bitmap");
    return run_sparse(w, d_res, true, d_qidx, res_len_bytes / 4, static_cast<cudaStream_t>(stream));
    API_END
}

abf_status abf_list_union_dense(const abf_worker* w, uint32_t* d_res, void* stream) {
    API_BEGIN
    if (!w || w->kind == 0 || w->batch != 1) return fail(ABF_ERR_INVALID, "abf_list_union_dense needs a dense worker of one query");
    return run_dense(w, d_res, n_words_of(w->ix->n_ads), static_cast<cudaStream_t>(stream));
    API_END
}

abf_status abf_batch_list_union_dense(const abf_worker* w, uint32_t* d_res, uint32_t res_len_u32, void* stream) {
    API_BEGIN
    if (!w || w->kind == 0) return fail(ABF_ERR_INVALID, "abf_batch_list_union_dense needs a dense worker");
    if (w->batch > 1 && uint64_t(res_len_u32) * 32 < w->ix->n_ads)
        return fail(ABF_ERR_INVALID, "res_len_u32 smaller than the bitmap");
    return run_dense(w, d_res, res_len_u32, static_cast<cudaStream_t>(stream));
    API_END
}

abf_status abf_collect_ids(abf_index* ix, const uint32_t* d_bitmap, uint64_t n_bits, uint32_t* d_ids,
                           uint64_t ids_capacity, uint64_t* d_count, void* stream) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!d_bitmap || !d_count || (ids_capacity && !d_ids)) return fail(ABF_ERR_INVALID, "abf_collect_ids: bad arguments");
    if (n_bits == 0 || n_bits > (1ull << 32)) return fail(ABF_ERR_RANGE, "n_bits must be in [1, 2^32]");
    CUDA_TRY(cudaSetDevice(ix->device));
    abf_workspace* ws = nullptr;
    ABF_TRY(own_ws(ix, 1, 1, n_bits, &ws));
    abf::CompactArgs ca{};
    ca.bm = d_bitmap;
    ca.stride = n_words_of(n_bits);
    ca.n_q = 1;
    ca.n_bits = n_bits;
    ca.n_chunks = abf::compact_chunks(n_bits);
    ca.status = ws->scan_status;
    ca.ticket = ws->ticket;
    ca.ids = d_ids;
    ca.capacity = ids_capacity;
    ca.id_offsets = ws->id_off;
    ca.id_counts = d_count;
    ca.err = ws->err;
    ca.spin_limit = ws->spin_limit;
    ABF_TRY(run_compact(ix, ca, static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

abf_status abf_batch_collect_ids(abf_index* ix, abf_workspace* ws, const uint32_t* d_bitmaps, uint64_t stride_words,
                                 uint32_t n_bitmaps, uint32_t* d_ids, uint64_t ids_capacity, uint64_t* d_id_offsets,
                                 void* stream) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!ws || ws->ix != ix || !d_id_offsets || (n_bitmaps && !d_bitmaps) || (ids_capacity && !d_ids))
        return fail(ABF_ERR_INVALID, "abf_batch_collect_ids: bad arguments");
    if (n_bitmaps == 0) return ABF_OK;
    if (n_bitmaps > ws->max_q) return fail(ABF_ERR_CAPACITY, "abf_batch_collect_ids: more bitmaps than the workspace's queries");
    const uint64_t n_words = n_words_of(ix->n_ads);
    if (stride_words < n_words) return fail(ABF_ERR_INVALID, "abf_batch_collect_ids: stride_words < (n_ads+31)/32");
    CUDA_TRY(cudaSetDevice(ix->device));
    abf::CompactArgs ca{};
    ca.bm = d_bitmaps;
    ca.stride = stride_words;
    ca.n_q = n_bitmaps;
    ca.n_bits = ix->n_ads;
    ca.n_chunks = abf::compact_chunks(ix->n_ads);
    ca.status = ws->scan_status;
    ca.ticket = ws->ticket;
    ca.ids = d_ids;
    ca.capacity = d_ids ? ids_capacity : 0;
    ca.id_offsets = d_id_offsets;
    ca.id_counts = nullptr;
    ca.err = ws->err;
    ca.spin_limit = ws->spin_limit;
    ABF_TRY(run_compact(ix, ca, static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

// ---------------------------------------------------------------------------
// native batch API
// ---------------------------------------------------------------------------
abf_status abf_workspace_create(abf_index* ix, uint32_t max_queries, uint64_t max_terms, abf_workspace** out) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!out || max_queries == 0) return fail(ABF_ERR_INVALID, "abf_workspace_create: bad arguments");
    CUDA_TRY(cudaSetDevice(ix->device));
    *out = nullptr;
    abf_workspace* w = new abf_workspace();
    abf_status st = ws_alloc(ix, max_queries, std::max<uint64_t>(max_terms, 1), ix->n_ads, w);
    if (st != ABF_OK) {
        delete w;
        return st;
    }
    *out = w;
    return ABF_OK;
    API_END
}

}  // extern "C"

namespace abf {
const uint8_t* ws_paths(const abf_workspace* w) { return w->path_out; }
uint32_t* ws_err(abf_workspace* w) { return w->err; }
}  // namespace abf

extern "C" {

abf_status abf_workspace_free(abf_workspace* w) {
    API_BEGIN
    if (!w) return ABF_OK;
    if (w->ix && w->ix->on_device) {
        cudaSetDevice(w->ix->device);
        cudaDeviceSynchronize();
    }
    ws_release(w);
    delete w;
    return ABF_OK;
    API_END
}

abf_status abf_workspace_check(abf_workspace* w, void* stream) {
    API_BEGIN
    if (!w) return fail(ABF_ERR_INVALID, "null workspace");
    CUDA_TRY(cudaSetDevice(w->ix->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t err = 0;
    CUDA_TRY(cudaMemcpyAsync(&err, w->err, 4, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    CUDA_TRY(cudaMemsetAsync(w->err, 0, 4, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (err & abf::kErrTermRange) return fail(ABF_ERR_CAPACITY, "a query's term offsets exceed the workspace's max_terms");
    if (err) return fail(ABF_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(err) + ")");
    return ABF_OK;
    API_END
}

abf_status abf_workspace_paths(abf_workspace* w, uint8_t* h_paths, uint32_t n, void* stream) {
    API_BEGIN
    if (!w || (n && !h_paths)) return fail(ABF_ERR_INVALID, "abf_workspace_paths: bad arguments");
    if (n > w->max_q) return fail(ABF_ERR_CAPACITY, "abf_workspace_paths: more queries than the workspace holds");
    if (n == 0) return ABF_OK;
    CUDA_TRY(cudaSetDevice(w->ix->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CUDA_TRY(cudaMemcpyAsync(h_paths, w->path_out, n, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return ABF_OK;
    API_END
}

abf_status abf_workspace_set_wait_limit(abf_workspace* w, uint32_t polls) {
    if (!w || polls == 0) return fail(ABF_ERR_INVALID, "abf_workspace_set_wait_limit: null workspace or zero polls");
    w->spin_limit = polls;
    return ABF_OK;
}

abf_status abf_workspace_selftest_waits(abf_workspace* w, uint32_t polls, void* stream) {
    API_BEGIN
    if (!w || polls == 0) return fail(ABF_ERR_INVALID, "abf_workspace_selftest_waits: null workspace or zero polls");
    CUDA_TRY(cudaSetDevice(w->ix->device));
    // the first two look-back words of the compaction scratch (a workspace
    // has one per chunk of every query, plus one)
    CUDA_TRY(abf::launch_wait_selftest(w->scan_status, w->err, polls, static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

abf_status abf_batch_run(abf_index* ix, abf_workspace* ws, const abf_batch* b, void* stream) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!ws || !b || ws->ix != ix) return fail(ABF_ERR_INVALID, "abf_batch_run: bad arguments");
    if (b->n_queries && (!b->d_terms || !b->d_offsets || !b->d_bitmaps))
        return fail(ABF_ERR_INVALID, "abf_batch_run: null device array");
    return run_batch(ix, ws, b, RunOpts{}, static_cast<cudaStream_t>(stream));
    API_END
}

}  // extern "C"

struct abf_batch_graph {
    abf_index* ix = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t n_kernel_nodes = 0;
};

extern "C" {

abf_status abf_batch_graph_create(abf_index* ix, abf_workspace* ws, const abf_batch* b, void* stream,
                                  abf_batch_graph** out) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!ws || !b || !out || ws->ix != ix) return fail(ABF_ERR_INVALID, "abf_batch_graph_create: bad arguments");
    if (!stream) return fail(ABF_ERR_INVALID, "abf_batch_graph_create: capture needs a created stream, not the default one");
    if (b->n_queries == 0) return fail(ABF_ERR_INVALID, "abf_batch_graph_create: empty batch");
    if (!b->d_terms || !b->d_offsets || !b->d_bitmaps) return fail(ABF_ERR_INVALID, "abf_batch_graph_create: null device array");
    *out = nullptr;
    CUDA_TRY(cudaSetDevice(ix->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // one direct run first: it makes every host-side setting the batch needs
    // (kernel attributes, the dense bitmaps' tensor maps), so that the
    // captured run issues only stream work; no event records in the graph
    const bool prof = ix->prof_on;
    ix->prof_on = false;
    abf_status st = run_batch(ix, ws, b, RunOpts{}, s);
    if (st != ABF_OK) {
        ix->prof_on = prof;
        return st;
    }
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        ix->prof_on = prof;
        return fail(ABF_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
    }
    st = run_batch(ix, ws, b, RunOpts{}, s);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(s, &graph);  // always ends the capture, also after a failed run
    ix->prof_on = prof;
    if (st != ABF_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return fail(ABF_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(ABF_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    auto* g = new abf_batch_graph();
    g->ix = ix;
    g->graph = graph;
    g->exec = exec;
    size_t n_nodes = 0;
    if (cudaGraphGetNodes(graph, nullptr, &n_nodes) == cudaSuccess && n_nodes) {
        std::vector<cudaGraphNode_t> nodes(n_nodes);
        if (cudaGraphGetNodes(graph, nodes.data(), &n_nodes) == cudaSuccess)
            for (size_t i = 0; i < n_nodes; ++i) {
                cudaGraphNodeType ty;
                if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel)
                    ++g->n_kernel_nodes;
            }
    }
    *out = g;
    return ABF_OK;
    API_END
}

abf_status abf_batch_graph_replay(abf_batch_graph* g, void* stream) {
    API_BEGIN
    if (!g) return fail(ABF_ERR_INVALID, "null graph");
    CUDA_TRY(cudaSetDevice(g->ix->device));
    CUDA_TRY(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
    abf::count_launch(g->n_kernel_nodes);
    return ABF_OK;
    API_END
}

abf_status abf_batch_graph_kernels(const abf_batch_graph* g, uint32_t* n_out) {
    if (!g || !n_out) return fail(ABF_ERR_INVALID, "null argument");
    *n_out = g->n_kernel_nodes;
    return ABF_OK;
}

abf_status abf_batch_graph_destroy(abf_batch_graph* g) {
    API_BEGIN
    if (!g) return ABF_OK;
    cudaSetDevice(g->ix->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return ABF_OK;
    API_END
}

abf_status abf_query(abf_index* ix, const uint32_t* terms, uint32_t n_terms, abf_path path, uint32_t* d_bitmap,
                     uint32_t* d_ids, uint64_t ids_capacity, uint64_t* d_count, void* stream) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!d_bitmap || (n_terms && !terms) || (d_ids && !d_count))
        return fail(ABF_ERR_INVALID, "abf_query: bad arguments");
    CUDA_TRY(cudaSetDevice(ix->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    abf_workspace* ws = nullptr;
    ABF_TRY(own_ws(ix, 1, n_terms, ix->n_ads, &ws));
    const size_t need = size_t(n_terms) * 4 + 16;
    if (!ix->stage_event) {
        cudaEvent_t ev;
        CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        ix->stage_event = ev;
    }
    cudaEvent_t ev = static_cast<cudaEvent_t>(ix->stage_event);
    CUDA_TRY(cudaEventSynchronize(ev));  // the previous upload has left the staging buffer
    if (ix->h_stage_bytes < need) {
        if (ix->h_stage) cudaFreeHost(ix->h_stage);
        ix->h_stage = nullptr;
        ix->h_stage_bytes = 0;
        CUDA_TRY(cudaMallocHost(&ix->h_stage, std::max<size_t>(need, 4096)));
        ix->h_stage_bytes = std::max<size_t>(need, 4096);
    }
    uint64_t* off = static_cast<uint64_t*>(ix->h_stage);
    off[0] = 0;
    off[1] = n_terms;
    if (n_terms) std::memcpy(off + 2, terms, size_t(n_terms) * 4);
    CUDA_TRY(cudaMemcpyAsync(ws->q_off, off, 16, cudaMemcpyHostToDevice, s));
    if (n_terms) CUDA_TRY(cudaMemcpyAsync(ws->q_terms, off + 2, size_t(n_terms) * 4, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaEventRecord(ev, s));
    abf_batch b{};
    b.d_terms = ws->q_terms;
    b.d_offsets = ws->q_off;
    b.n_queries = 1;
    b.path = path;
    b.d_bitmaps = d_bitmap;
    b.bitmap_stride_words = round4(n_words_of(ix->n_ads));
    b.d_ids = d_ids;
    b.ids_capacity = d_ids ? ids_capacity : 0;
    b.d_id_offsets = ws->id_off;
    RunOpts ro;
    ro.id_counts = d_count;
    return run_batch(ix, ws, &b, ro, s);
    API_END
}

abf_status abf_index_list_bytes(const abf_index* ix, uint64_t* h_out, uint32_t n) {
    if (!ix || !h_out || n < ix->n_terms) return fail(ABF_ERR_INVALID, "abf_index_list_bytes: bad arguments");
    std::memcpy(h_out, ix->h_term_bytes.data(), size_t(ix->n_terms) * 8);
    return ABF_OK;
}

abf_status abf_planner_features(abf_index* ix, const uint32_t* d_terms, const uint64_t* d_offsets, uint32_t n_q,
                                float* d_features, void* stream) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (n_q && (!d_terms || !d_offsets || !d_features)) return fail(ABF_ERR_INVALID, "abf_planner_features: null pointer");
    CUDA_TRY(cudaSetDevice(ix->device));
    CUDA_TRY(abf::launch_planner(abf::view_of(ix), nullptr, d_terms, d_offsets, n_q, ix->tuning.heavy_min_len,
                                 ix->n_postings, d_features, nullptr, nullptr, static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

abf_status abf_planner_set(abf_index* ix, const float* h_params) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    CUDA_TRY(cudaSetDevice(ix->device));
    if (!h_params) {
        CUDA_TRY(cudaDeviceSynchronize());
        dev_free(ix->dev.planner);
        return ABF_OK;
    }
    if (!ix->dev.planner) ABF_TRY(dev_alloc(&ix->dev.planner, ABF_PLANNER_PARAMS));
    CUDA_TRY(cudaMemcpy(ix->dev.planner, h_params, sizeof(float) * ABF_PLANNER_PARAMS, cudaMemcpyHostToDevice));
    return ABF_OK;
    API_END
}

abf_status abf_planner_predict(abf_index* ix, const uint32_t* d_terms, const uint64_t* d_offsets, uint32_t n_q,
                               float* d_pred, uint8_t* d_paths, void* stream) {
    API_BEGIN
    ABF_TRY(need_device(ix));
    if (!ix->dev.planner) return fail(ABF_ERR_STATE, "no planner parameters installed (abf_planner_set)");
    if (n_q && (!d_terms || !d_offsets)) return fail(ABF_ERR_INVALID, "abf_planner_predict: null pointer");
    CUDA_TRY(cudaSetDevice(ix->device));
    CUDA_TRY(abf::launch_planner(abf::view_of(ix), ix->dev.planner, d_terms, d_offsets, n_q, ix->tuning.heavy_min_len,
                                 ix->n_postings, nullptr, d_pred, d_paths, static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

abf_status abf_mlp_forward(const float* d_params, const float* d_x, uint32_t n, float* d_y, void* stream) {
    API_BEGIN
    if (!d_params || (n && (!d_x || !d_y))) return fail(ABF_ERR_INVALID, "abf_mlp_forward: null pointer");
    CUDA_TRY(abf::launch_mlp_forward(d_params, d_x, n, d_y, static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

abf_status abf_mlp_grad(const float* d_params, const float* d_x, const float* d_t, const float* d_mask, uint32_t n,
                        float* d_grad, float* d_loss, void* stream) {
    API_BEGIN
    if (!d_params || !d_grad || !d_loss || (n && (!d_x || !d_t || !d_mask)))
        return fail(ABF_ERR_INVALID, "abf_mlp_grad: null pointer");
    CUDA_TRY(abf::launch_mlp_grad(d_params, d_x, d_t, d_mask, n, d_grad, d_loss, static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

abf_status abf_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, uint32_t step, float lr,
                        float beta1, float beta2, float eps, void* stream) {
    API_BEGIN
    if (!d_params || !d_grad || !d_m || !d_v) return fail(ABF_ERR_INVALID, "abf_mlp_adam: null pointer");
    CUDA_TRY(abf::launch_adam(d_params, d_grad, d_m, d_v, step, lr, beta1, beta2, eps,
                              static_cast<cudaStream_t>(stream)));
    return ABF_OK;
    API_END
}

abf_status abf_index_list_flags(const abf_index* ix, uint32_t* h_out, uint32_t n) {
    if (!ix || !h_out || n < ix->n_terms) return fail(ABF_ERR_INVALID, "abf_index_list_flags: bad arguments");
    const auto& d = ix->derived;
    for (uint32_t t = 0; t < ix->n_terms; ++t)
        h_out[t] = (d.term_dense[t] != abf::kNone ? ABF_LIST_DENSE : 0u) |
                   (d.term_dir[t] != abf::kNone ? ABF_LIST_DIRECTORY : 0u);
    return ABF_OK;
}

abf_status abf_profile_enable(abf_index* ix, int on) {
    API_BEGIN
    if (!ix) return fail(ABF_ERR_INVALID, "null index");
    if (on && !ix->prof) ix->prof = new Profiler();
    ix->prof_on = on != 0;
    return ABF_OK;
    API_END
}

abf_status abf_profile_read(abf_index* ix, abf_kernel_time* out, uint32_t cap, uint32_t* n_out) {
    API_BEGIN
    if (!ix || !n_out || (cap && !out)) return fail(ABF_ERR_INVALID, "abf_profile_read: bad arguments");
    uint64_t launches[K_NKERNELS] = {};
    double ms[K_NKERNELS] = {};
    if (ix->prof) {
        auto* p = static_cast<Profiler*>(ix->prof);
        for (auto& r : p->recs) {
            CUDA_TRY(cudaEventSynchronize(r.b));
            float e = 0;
            CUDA_TRY(cudaEventElapsedTime(&e, r.a, r.b));
            ms[r.kid] += e;
            launches[r.kid] += 1;
            p->pool.push_back(r.a);
            p->pool.push_back(r.b);
        }
        p->recs.clear();
    }
    uint32_t k = 0;
    for (int i = 0; i < K_NKERNELS; ++i) {
        if (!launches[i]) continue;
        if (k < cap) {
            std::memset(out[k].name, 0, sizeof(out[k].name));
            std::strncpy(out[k].name, kKernelNames[i], sizeof(out[k].name) - 1);
            out[k].launches = launches[i];
            out[k].total_ms = ms[i];
        }
        ++k;
    }
    *n_out = k;
    return ABF_OK;
    API_END
}

}  // extern "C"
