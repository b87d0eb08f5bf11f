/*
 * adabool.h -- C ABI of the B200 Boolean-filtering engine (libadabool.so).
 *
 * A filter matrix is a set of (term, ad) pairs. A query is a set of terms;
 * its match set is the OR-union of the posting lists of its terms, returned
 * as a bitmap over ads (word v>>5, bit v&31 -- the layout the reference's
 * kernels write and CollectIdsFromBitmap reads, test/adsfilter_batch.cu:82-97)
 * and, optionally, as an ascending list of uint32 ad IDs.
 *
 * Conventions (all entry points):
 *   - every function returns abf_status; nothing aborts and no C++ exception
 *     crosses this boundary; abf_last_error_string() describes the last
 *     failure on the calling thread;
 *   - pointers named d_* are device pointers on the index's device; h_*
 *     and plain pointers are host pointers;
 *   - stream arguments are cudaStream_t passed as void* (0 = legacy default);
 *     all device work is enqueued on that stream and the call returns
 *     without synchronising unless its comment says otherwise;
 *   - an index or worker is used by one stream at a time (the reference has
 *     the same rule: one caller stream, no internal locks).
 *
 * Each entry point names the reference interface it replaces as
 * file:line within the reference project (yxr620/AdaBool).
 */
#ifndef ADABOOL_H_
#define ADABOOL_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ABF_ABI_VERSION 2u
/* postings per compressed block of the list format */
#define ABF_BLOCK_POSTINGS 128u

typedef enum abf_status {
    ABF_OK = 0,
    ABF_ERR_INVALID = 1,   /* bad argument (null pointer, zero size, ...) */
    ABF_ERR_RANGE = 2,     /* a term or ad id outside the declared domain */
    ABF_ERR_CUDA = 3,      /* a CUDA runtime call failed */
    ABF_ERR_OOM = 4,       /* host or device allocation failed */
    ABF_ERR_STATE = 5,     /* object not in a state that allows the call */
    ABF_ERR_IO = 6,        /* file read/write failed or bad file format */
    ABF_ERR_TIMEOUT = 7,   /* a bounded device-side wait gave up */
    ABF_ERR_CAPACITY = 8,  /* output larger than the capacity given */
    ABF_ERR_INTERNAL = 9
} abf_status;

/* Which kernel family answers a query. */
typedef enum abf_path {
    ABF_PATH_AUTO = 0,    /* planner decides per query (learned, else fixed rule) */
    ABF_PATH_PROBE = 1,   /* bitmap-probe: scan every block, test the query's term bitmap */
    ABF_PATH_UNION = 2,   /* list-union: decode only the query's lists, scatter to the bitmap */
    ABF_PATH_HYBRID = 3,  /* long lists merged tile by tile in shared memory, short lists scattered */
    ABF_PATH_TILE = 4     /* every list merged tile by tile (HYBRID with threshold 0) */
} abf_path;

typedef struct abf_index abf_index;
typedef struct abf_workspace abf_workspace;
typedef struct abf_worker abf_worker;

/* ------------------------------------------------------------------ */
/* Index build / free / persistence                                    */
/* ------------------------------------------------------------------ */

enum {
    ABF_BUILD_HOST_ONLY = 1u << 0, /* keep the index on the host; no device needed */
    ABF_BUILD_KEEP_HOST = 1u << 1  /* keep a host copy after the upload */
};

typedef struct abf_build_opts {
    int device;          /* CUDA device ordinal (ignored with ABF_BUILD_HOST_ONLY) */
    uint32_t flags;      /* ABF_BUILD_* */
    int n_threads;       /* host threads for the build; <= 0 = all cores */
    uint32_t dense_div;  /* a list with len * dense_div >= n_ads also gets a dense
                            bitmap, merged without decoding; 0 = 128, 0xffffffff = none */
} abf_build_opts;

typedef struct abf_index_stats {
    uint32_t n_terms;
    uint32_t n_ads;
    uint64_t n_postings;        /* unique (term, ad) pairs */
    uint64_t n_blocks;          /* compressed blocks */
    uint64_t payload_bytes;     /* bit-packed gap bytes */
    uint64_t device_bytes;      /* all device arrays of the index */
    uint32_t max_list_len;
    uint32_t on_device;         /* 1 if the device copy exists */
    uint32_t n_dense_lists;     /* lists that also have a dense bitmap */
    uint32_t n_directory_lists; /* lists with a per-tile block directory */
    uint64_t dense_bytes;       /* bytes of the dense bitmaps */
} abf_index_stats;

/* Build from COO pairs (terms[i], ads[i]), i < nnz. Pairs may be in any
 * order; duplicates are merged. Every term must be < n_terms and every ad
 * < n_ads, else ABF_ERR_RANGE. Replaces ivf_list::BuildFrom
 * (src/AdaBool/inverted_list.h:348-374) and the per-block key metadata it
 * derives (src/AdaBool/inverted_list.h:90-148). */
abf_status abf_index_build_coo(const uint32_t* terms, const uint32_t* ads, uint64_t nnz,
                               uint32_t n_terms, uint32_t n_ads,
                               const abf_build_opts* opts, abf_index** out);

/* Build from CSR: the postings of term t are ads[offsets[t] .. offsets[t+1]),
 * offsets has n_terms+1 entries. Lists need not be sorted or unique. Same
 * replacement as abf_index_build_coo, without the COO grouping step
 * (src/AdaBool/inverted_list.h:351-355). */
abf_status abf_index_build_csr(const uint64_t* offsets, const uint32_t* ads,
                               uint32_t n_terms, uint32_t n_ads,
                               const abf_build_opts* opts, abf_index** out);

/* Frees the index and its device arrays (synchronises the device). The
 * reference frees through LenBuffer destructors (src/AdaBool/len_buffer.h:196-230). */
abf_status abf_index_free(abf_index* index);

abf_status abf_index_get_stats(const abf_index* index, abf_index_stats* out);

/* Per-term list lengths (n_terms entries) into a host array. */
abf_status abf_index_list_lengths(const abf_index* index, uint32_t* h_out, uint32_t n);

/* Decode the list of one term on the host from the compressed arrays
 * (needs the host copy: ABF_BUILD_HOST_ONLY or ABF_BUILD_KEEP_HOST).
 * *n_out receives the list length; at most cap ids are written. */
abf_status abf_index_decode_list(const abf_index* index, uint32_t term,
                                 uint32_t* h_ids, uint64_t cap, uint64_t* n_out);

/* Binary index file: one header plus the compressed arrays, loaded with a
 * single host read and one upload per array. No reference counterpart: the
 * reference rebuilds from text COO on every run (test/adsfilter_q_all.cu:127-161). */
abf_status abf_index_save(const abf_index* index, const char* path);
abf_status abf_index_load(const char* path, const abf_build_opts* opts, abf_index** out);

/* Upload a host-only index to a device. */
abf_status abf_index_to_device(abf_index* index, int device);

/* ------------------------------------------------------------------ */
/* Kernel tuning                                                       */
/* ------------------------------------------------------------------ */

typedef struct abf_tuning {
    uint32_t tile_words;      /* words per merge tile: a power of two, 256 .. 16384 */
    uint32_t warps_per_tile;  /* warps that share one tile's lists: 1, 2, 4 or 8 */
    uint32_t heavy_min_len;   /* HYBRID: lists with >= this many postings are merged
                                 per tile, shorter lists are scattered */
    uint32_t probe_chunk_blocks; /* blocks per CTA in the bitmap-probe scan */
    uint32_t scatter_blocks_per_warp; /* consecutive blocks a union warp takes */
    uint32_t ctas_per_sm;     /* grid = SMs x this, for the persistent kernels */
    uint32_t probe_cap;       /* queries of one batch that may take the probe path (<= 65536) */
    float probe_min_fraction; /* fixed rule (ABF_PATH_AUTO without a planner): probe
                                 when the query's lists hold more than this fraction
                                 of all blocks, else HYBRID or list-union (below) */
    uint32_t group_min_queries; /* batches of at least this many queries merge the
                                 dense bitmaps of all their dense-only queries in one
                                 pass per 64- or 32-word tile (each tile's slice of every
                                 dense bitmap staged once in shared memory by TMA, then
                                 ORed per query); needs at most 767 dense bitmaps;
                                 0 = never */
    uint32_t fixed_tile_shape;  /* 0: a batch too small to fill the GPU at tile_words x
                                 warps_per_tile runs the merge kernel with 8-warp CTAs
                                 and tiles narrowed down to 1,024 words; 1: always the
                                 given shape */
    uint32_t fixed_hybrid_min_len; /* fixed rule: a query that does not probe takes HYBRID
                                 when one of its lists has at least this many postings,
                                 else list-union; 0 = never HYBRID. Default
                                 ceil(33 * n_ads / 256): the density at which the
                                 reference stores a 256-id bucket as a bitset
                                 (src/AdaBool/inverted_list.h:425-458) */
    uint32_t compact_ctas_per_sm; /* resident warps per SM of the compaction, in eights
                                 (1..6, default 6 = 48 warps, 12 CTAs of 4 warps);
                                 fewer leave room for another stream's kernels */
    uint32_t group_tile_words;  /* dense group kernel tile: 0 or 64 = 64 words wherever
                                 one stage fits shared memory (two stages where they
                                 fit; the window's lists read from global memory when
                                 they do not fit beside the stage), else 32; 32 =
                                 always 32 */
} abf_tuning;

abf_status abf_get_tuning(const abf_index* index, abf_tuning* out);
abf_status abf_set_tuning(abf_index* index, const abf_tuning* t);

/* Rebuilds the dense bitmaps (and block directory) for a new dense_div
 * (see abf_build_opts; 0xffffffff = none) and re-uploads them; synchronises
 * the device. The merge threshold heavy_min_len is left as it is. */
abf_status abf_index_set_dense_div(abf_index* index, uint32_t dense_div);

/* ------------------------------------------------------------------ */
/* Reference-shaped operator API (prepare a worker, run it into d_res)  */
/* ------------------------------------------------------------------ */
/* These keep the reference's contract: d_res is caller-owned and the
 * kernels OR into it, so a caller that zeroes d_res gets exactly the match
 * set; the bitmap has (n_ads + 31) / 32 words per query. */

/* Sparse worker for one query (or a flattened batch of queries) given as
 * host term ids; terms >= n_terms are ignored. Replaces
 * ivf_list::Prepare(keys) (src/AdaBool/inverted_list.h:481-527) together
 * with InvertedListWorker::Prepare / LoadBalanceTransformer::Prepare
 * (src/AdaBool/inverted_list.h:183-189, src/AdaBool/load_balance_transformer.h:50-69). */
abf_status abf_prepare_sparse(abf_index* index, const uint32_t* keys, uint64_t n_keys,
                              abf_worker** out);

/* Dense worker for one query given as a host term bitmap of len bytes
 * (bit t of byte t/8 set = term t in the query). Replaces
 * ivf_list::Prepare(len, bitmap) (src/AdaBool/inverted_list.h:530-543). */
abf_status abf_prepare_dense(abf_index* index, uint64_t len, const uint8_t* query_bitmap,
                             abf_worker** out);

/* Dense worker for batch_size queries whose term bitmaps are laid out
 * query-major, len bytes each (len a multiple of 4). Host variant replaces
 * ivf_list::PrepareBatch (src/AdaBool/inverted_list.h:564-574); the device
 * variant replaces PrepareBatchDevice (src/AdaBool/inverted_list.h:591-605)
 * and does not copy d_query_bitmap, which must outlive the worker. */
abf_status abf_prepare_batch(abf_index* index, uint64_t batch_size, uint64_t len,
                             const uint8_t* query_bitmap, abf_worker** out);
abf_status abf_prepare_batch_device(abf_index* index, uint64_t batch_size, uint64_t len,
                                    const uint8_t* d_query_bitmap, abf_worker** out);

abf_status abf_worker_free(abf_worker* worker);

/* Union of the sparse worker's lists ORed into d_res. Replaces
 * ListUnion_sparse (test/adsfilter_q_all.cu:64-105). */
abf_status abf_list_union_sparse(const abf_worker* worker, uint32_t* d_res, void* stream);

/* Bitmap-probe of the dense worker ORed into d_res. Replaces
 * ListUnion_dense (test/adsfilter_q_all.cu:26-61). */
abf_status abf_list_union_dense(const abf_worker* worker, uint32_t* d_res, void* stream);

/* Batched bitmap-probe: query b ORs into d_res + b * res_len_u32. Any batch
 * size (the reference stops at 32). Replaces BatchListUnion_dense
 * (test/adsfilter_batch.cu:28-36) and InvertedListBatchWorkerImpl::RunArrays
 * (src/AdaBool/inverted_list.cu.h:224-228). */
abf_status abf_batch_list_union_dense(const abf_worker* worker, uint32_t* d_res,
                                      uint32_t res_len_u32, void* stream);

/* Batched list-union: key i of the sparse worker ORs into
 * d_res + d_qidx[i] * (res_len_bytes / 4). Replaces BatchListUnion_sparse
 * (test/adsfilter_batch.cu:39-79). */
abf_status abf_batch_list_union_sparse(const abf_worker* worker, uint32_t* d_res,
                                       const uint32_t* d_qidx, uint32_t res_len_bytes,
                                       void* stream);

/* Ascending ids of the set bits below n_bits of a device bitmap, written
 * to d_ids (at most ids_capacity), the count to *d_count (device). Replaces
 * the host-side CollectIdsFromBitmap (test/adsfilter_q_all.cu:108-119,
 * test/adsfilter_batch.cu:82-97). Uses a workspace of the index. */
abf_status abf_collect_ids(abf_index* index, const uint32_t* d_bitmap, uint64_t n_bits,
                           uint32_t* d_ids, uint64_t ids_capacity, uint64_t* d_count,
                           void* stream);

/* Ascending ids of a batch of n_bitmaps device bitmaps (bitmap q at
 * d_bitmaps + q * stride_words, (n_ads + 31) / 32 words each, bits past n_ads
 * ignored), packed into d_ids: bitmap q's ids at d_id_offsets[q] ..
 * d_id_offsets[q+1] (n_bitmaps + 1 offsets, written); ids past ids_capacity
 * are not written, the offsets stay exact. One pass per bitmap (count, offset
 * by look-back, write), with the workspace's compaction scratch (not
 * concurrently with a batch on the same workspace); n_bitmaps at most the
 * workspace's max_queries. Replaces the host loop of CollectIdsFromBitmap over
 * a batch's results (test/adsfilter_batch.cu:82-97,512-519). */
abf_status abf_batch_collect_ids(abf_index* index, abf_workspace* ws, const uint32_t* d_bitmaps,
                                 uint64_t stride_words, uint32_t n_bitmaps, uint32_t* d_ids,
                                 uint64_t ids_capacity, uint64_t* d_id_offsets, void* stream);

/* Allocation-free variant of abf_collect_ids, with no counterpart in the
 * reference. For callers that may not allocate device memory when they
 * need the ids: an engine that owns all device memory and forbids plugins
 * to allocate, a serving thread that cannot afford cudaMalloc's possible
 * device-wide synchronisation, code that must not hit out-of-memory in
 * the middle of a request. Needs no index and calls no cudaMalloc/cudaFree:
 * its scratch is one static device array (about 256 KB per device, kept
 * until the process exits) sized for at most ABF_NOALLOC_MAX_BITS bits.
 * Larger bitmaps are refused with ABF_ERR_CAPACITY -- where abf_collect_ids
 * refuses only bitmaps above 2^32 bits, with ABF_ERR_RANGE. The first call
 * on a device looks up that array's device address (cudaGetSymbolAddress)
 * and should come before any stream capture. Every call on a device shares
 * the array: calls whose work can overlap on the GPU race and must be
 * ordered by the caller (one stream, or events). Ids and count equal
 * abf_collect_ids's. A device-side wait that gave up is reported by
 * abf_collect_ids_noalloc_check, not by this call's return value. */
#define ABF_NOALLOC_MAX_BITS (1ull << 30)
abf_status abf_collect_ids_noalloc(const uint32_t* d_bitmap, uint64_t n_bits, uint32_t* d_ids,
                                   uint64_t ids_capacity, uint64_t* d_count, void* stream);
/* Synchronises `stream` and reports the error word that the last
 * abf_collect_ids_noalloc call on the current device left: ABF_ERR_TIMEOUT
 * if its look-back wait gave up (its ids are then not valid), else ABF_OK.
 * Each abf_collect_ids_noalloc call clears the word first. */
abf_status abf_collect_ids_noalloc_check(void* stream);

/* ------------------------------------------------------------------ */
/* Native batched API (no reference counterpart beyond the batch paths) */
/* ------------------------------------------------------------------ */

/* A workspace holds the scratch arrays of one in-flight batch: planning
 * tables, probe bitmaps, compaction counts, an error flag. Sized for at
 * most max_queries queries and max_terms query terms in total. */
abf_status abf_workspace_create(abf_index* index, uint32_t max_queries, uint64_t max_terms,
                                abf_workspace** out);
abf_status abf_workspace_free(abf_workspace* ws);
/* Reads and clears the device error flag (synchronises the stream):
 * ABF_ERR_TIMEOUT when a bounded device wait gave up, ABF_ERR_CAPACITY when a
 * query's term offsets exceeded the workspace. */
abf_status abf_workspace_check(abf_workspace* ws, void* stream);

/* The abf_path each of the first n queries of the workspace's last batch ran
 * on (after the planner or the fixed rule resolved ABF_PATH_AUTO, and after
 * probe queries beyond probe_cap fell back to UNION), into a host array;
 * synchronises the stream. No reference counterpart. */
abf_status abf_workspace_paths(abf_workspace* ws, uint8_t* h_paths, uint32_t n, void* stream);

/* Bounded device waits. The kernels launched with this workspace poll a
 * compaction look-back word or an mbarrier at most `polls` times (default
 * 2^22, well over a second) before they give up, set the workspace's error
 * flag (abf_workspace_check then returns ABF_ERR_TIMEOUT) and return; no
 * kernel traps or spins without end. The reference has no device waits (its
 * kernels are launched back to back, test/adsfilter_q_all.cu:26-105). */
abf_status abf_workspace_set_wait_limit(abf_workspace* ws, uint32_t polls);

/* Diagnostic of those waits: launches, on `stream`, one CTA that arms an
 * mbarrier for a copy that is never issued and one that looks back at a
 * compaction status word that nothing publishes; both wait with the same
 * device code as the path kernels for at most `polls` polls, give up, set
 * their bits in the workspace's error flag and return. A following
 * abf_workspace_check returns ABF_ERR_TIMEOUT, and the context stays usable.
 * Uses the workspace's compaction scratch: not concurrently with a batch on
 * the same workspace. No reference counterpart. */
abf_status abf_workspace_selftest_waits(abf_workspace* ws, uint32_t polls, void* stream);

typedef struct abf_batch {
    const uint32_t* d_terms;     /* flat query terms (device) */
    const uint64_t* d_offsets;   /* n_queries + 1 offsets into d_terms (device) */
    uint32_t n_queries;
    const uint8_t* d_paths;      /* per-query abf_path (device) or NULL */
    abf_path path;               /* used when d_paths is NULL; AUTO = fixed rule per query */
    uint32_t* d_bitmaps;         /* n_queries x bitmap_stride_words output bitmaps, overwritten */
    uint64_t bitmap_stride_words;/* >= (n_ads + 31) / 32, a multiple of 4 */
    uint32_t* d_ids;             /* optional: packed ascending ids of every query */
    uint64_t ids_capacity;       /* entries available in d_ids */
    uint64_t* d_id_offsets;      /* optional (required with d_ids): n_queries + 1 */
} abf_batch;

/* Runs a batch: planning, merge tiles, scatter, probe and (with d_ids)
 * compaction, all on `stream`, no host synchronisation and no allocation,
 * so the call can be captured into a CUDA graph. Queries whose ids do not
 * fit ids_capacity get their offsets but ids are written only below the
 * capacity. */
abf_status abf_batch_run(abf_index* index, abf_workspace* ws, const abf_batch* batch,
                         void* stream);

/* A batch as one CUDA-graph launch. abf_batch_graph_create runs the batch
 * once on `stream` (it must be a created stream, not the legacy default),
 * then captures a second run into a CUDA graph and instantiates it: every
 * kernel and memset node of abf_batch_run (planner, plan, queue scan, probe
 * bits, dense group, merge tiles, scatter, probe, compaction). The graph
 * keeps the device pointers and the query count of *batch: each
 * abf_batch_graph_replay answers whatever terms, offsets and paths those
 * arrays hold when it runs, so a caller refills them on the stream and
 * replays (a shorter batch pads its offsets with empty queries). The index,
 * the workspace and the batch's arrays must outlive the graph, and a
 * workspace serves one graph or batch at a time. The arrays must hold a
 * valid batch at creation (the first run reads them). The reference
 * launches six kernels per query or per batch of at most 32 from the host
 * (src/AdaBool/inverted_list.cu.h:185-228, test/adsfilter_batch.cu:453-502);
 * this has no counterpart there. */
typedef struct abf_batch_graph abf_batch_graph;
abf_status abf_batch_graph_create(abf_index* index, abf_workspace* ws, const abf_batch* batch,
                                  void* stream, abf_batch_graph** out);
abf_status abf_batch_graph_replay(abf_batch_graph* graph, void* stream);
/* Kernel nodes in the graph (the launches one replay makes). */
abf_status abf_batch_graph_kernels(const abf_batch_graph* graph, uint32_t* n_out);
abf_status abf_batch_graph_destroy(abf_batch_graph* graph);

/* One query from host terms: bitmap (overwritten, (n_ads+31)/32 words) and,
 * if d_ids is not NULL, its ascending ids with the count in *d_count. Uses
 * the index's own workspace; the call returns after the terms were
 * uploaded, without waiting for the kernels. */
abf_status abf_query(abf_index* index, const uint32_t* terms, uint32_t n_terms, abf_path path,
                     uint32_t* d_bitmap, uint32_t* d_ids, uint64_t ids_capacity,
                     uint64_t* d_count, void* stream);

/* ------------------------------------------------------------------ */
/* Learned path planner (no reference counterpart: the reference runs  */
/* both paths on every query and has no selection rule)                */
/* ------------------------------------------------------------------ */
/* Per query, 16 features (term count, sum / max / mean / spread of list
 * lengths, compressed bytes, estimated output density, dense-list and
 * short-list counts, batch position and size, ...) feed an MLP
 * 16 -> 64 -> 64 -> 3 (ReLU, FP32) that predicts log(microseconds) of the
 * PROBE, UNION and HYBRID paths; the cheapest is taken. Parameter block
 * (ABF_PLANNER_PARAMS floats): mu[16], sd[16] (feature standardisation),
 * W1[64][16], b1[64], W2[64][64], b2[64], W3[3][64], b3[3]. */
#define ABF_PLANNER_FEATURES 16
#define ABF_PLANNER_HIDDEN 64
#define ABF_PLANNER_OUTPUTS 3
#define ABF_PLANNER_PARAMS (2 * 16 + 64 * 16 + 64 + 64 * 64 + 64 + 3 * 64 + 3)

/* Raw (unstandardised) features of a batch: n_queries x 16 floats. */
abf_status abf_planner_features(abf_index* index, const uint32_t* d_terms, const uint64_t* d_offsets,
                                uint32_t n_queries, float* d_features, void* stream);
/* Installs planner parameters (host array) on the index; NULL removes
 * them. With parameters installed, ABF_PATH_AUTO queries of abf_batch_run
 * and abf_query take the planner's choice instead of the fixed rule. */
abf_status abf_planner_set(abf_index* index, const float* h_params);
/* The fused feature + MLP kernel on its own: predictions (n x 3, may be
 * NULL) and chosen abf_path per query (may be NULL). */
abf_status abf_planner_predict(abf_index* index, const uint32_t* d_terms, const uint64_t* d_offsets,
                               uint32_t n_queries, float* d_pred, uint8_t* d_paths, void* stream);

/* Training kernels of the MLP on standardised features x (n x 16):
 * forward (y: n x 3), mean-squared-error gradient over the entries where
 * mask is non-zero (grad in the parameter layout, overwritten; d_loss
 * points to 2 floats: the loss and the number of entries counted), and one
 * Adam step. The mu/sd entries are never updated. */
abf_status abf_mlp_forward(const float* d_params, const float* d_x, uint32_t n, float* d_y, void* stream);
abf_status abf_mlp_grad(const float* d_params, const float* d_x, const float* d_t, const float* d_mask, uint32_t n,
                        float* d_grad, float* d_loss, void* stream);
abf_status abf_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, uint32_t step, float lr,
                        float beta1, float beta2, float eps, void* stream);

/* ------------------------------------------------------------------ */
/* Measurement                                                         */
/* ------------------------------------------------------------------ */

/* Compressed bytes of every term's list (n_terms entries): payload plus
 * 16 bytes of block metadata per block. No reference counterpart. */
abf_status abf_index_list_bytes(const abf_index* index, uint64_t* h_out, uint32_t n);

/* Per-term representation flags (n_terms entries): ABF_LIST_DENSE when the
 * list also has a dense bitmap of (n_ads + 31) / 32 words that the merge
 * kernel reads instead of its blocks, ABF_LIST_DIRECTORY when it has a
 * per-tile block directory. No reference counterpart. */
#define ABF_LIST_DENSE 1u
#define ABF_LIST_DIRECTORY 2u
abf_status abf_index_list_flags(const abf_index* index, uint32_t* h_out, uint32_t n);

/* Kernel timing. While enabled, every kernel this index launches is
 * bracketed by CUDA events on the stream it is launched on;
 * abf_profile_read synchronises those events, returns per-kernel launch
 * counts and total milliseconds, and clears them. No reference counterpart
 * (the reference times launch + synchronise with a host clock,
 * test/adsfilter_q_all.cu:421-425). */
typedef struct abf_kernel_time {
    char name[24];
    uint64_t launches;
    double total_ms;
} abf_kernel_time;
abf_status abf_profile_enable(abf_index* index, int on);
abf_status abf_profile_read(abf_index* index, abf_kernel_time* out, uint32_t cap, uint32_t* n_out);

/* ------------------------------------------------------------------ */
/* Serving loop (no reference counterpart: the reference answers one    */
/* query, or one batch of at most 32, per host call)                    */
/* ------------------------------------------------------------------ */
/* A server owns one host thread that batches submitted queries and runs
 * each batch through abf_batch_run on one of n_streams streams, so the
 * next batch is cut and launched while earlier ones run (continuous
 * batching):
 *   - admission: a batch takes one range of a device pool of budget_bytes,
 *     allocated when the server is created: n x bitmap_stride_words x 4
 *     bytes of bitmaps plus, with ABF_SERVE_IDS, 4 x min(n_ads, sum of the
 *     query's list lengths) bytes of id room per query. Queries are cut
 *     first-in first-out; the first one that does not fit the largest free
 *     extent waits, with everything behind it, until results are released;
 *   - batching: with nothing in flight, whatever waits is launched at once;
 *     otherwise a free stream takes a batch once the oldest waiting query
 *     has waited window_us, or max_batch_queries / max_batch_terms are
 *     reached;
 *   - results stay in the pool (bitmap and ascending ids, device memory)
 *     until abf_server_release. When a batch completes, its id room is
 *     trimmed to the ids written and, without ABF_SERVE_BITMAPS, its
 *     bitmaps are freed. A batch's range is returned to the pool when the
 *     last of its queries is released.
 * Every query's result is the same whatever batch it runs in. Submit, poll
 * and release may be called from any threads. Kernel timing
 * (abf_profile_enable) must be off on the index while a server runs. */
typedef struct abf_server abf_server;

#define ABF_SERVE_BITMAPS 1u    /* keep each query's bitmap in its result */
#define ABF_SERVE_IDS 2u        /* compute each query's ascending ids */

typedef struct abf_server_opts {
    uint64_t budget_bytes;       /* device pool for bitmaps and ids (default 40 GiB) */
    uint32_t window_us;          /* longest wait of the oldest query before a cut (default 100) */
    uint32_t max_batch_queries;  /* default 1024 */
    uint64_t max_batch_terms;    /* default 2^22; also the longest query accepted */
    uint32_t n_streams;          /* batches in flight, 1..8 (default 4) */
    abf_path path;               /* path of every query; AUTO = installed planner, else fixed rule */
    uint32_t outputs;            /* ABF_SERVE_BITMAPS | ABF_SERVE_IDS (default both) */
} abf_server_opts;

typedef struct abf_server_result {
    uint64_t ticket;
    uint64_t tag;                /* as given to abf_server_submit */
    int32_t status;              /* ABF_OK, or the error of the query's batch */
    uint32_t path;               /* abf_path the query ran on */
    const uint32_t* d_bitmap;    /* (n_ads+31)/32 words, device; NULL without ABF_SERVE_BITMAPS */
    const uint32_t* d_ids;       /* ascending ids, device; NULL without ABF_SERVE_IDS */
    uint64_t n_ids;
    uint64_t t_arrival_ns;       /* abf_clock_ns() times */
    uint64_t t_launch_ns;
    uint64_t t_done_ns;          /* when the server thread saw the batch complete */
    uint32_t batch_queries;      /* size of the batch it ran in */
    uint32_t pad_;
} abf_server_result;

typedef struct abf_server_stats {
    uint64_t submitted, completed, released, rejected;
    uint64_t batches, failed_batches;
    uint64_t waiting, in_flight_batches;
    uint64_t pool_bytes, reserved_bytes, peak_reserved_bytes;
    uint64_t admission_waits;    /* cuts that left a waiting query behind for lack of pool
                                    room, plus stretches with no room for the head query */
    uint64_t path_queries[5];    /* queries per abf_path taken */
    uint64_t max_batch_queries_seen;
} abf_server_stats;

/* Monotonic clock of the server, nanoseconds (CLOCK_MONOTONIC). */
uint64_t abf_clock_ns(void);
abf_status abf_server_default_opts(abf_server_opts* opts);
/* The index must be on a device and outlive the server. */
abf_status abf_server_create(abf_index* index, const abf_server_opts* opts, abf_server** out);
/* Copies the terms; arrival_ns 0 = now. Term ids >= n_terms match
 * nothing (as in abf_query). ABF_ERR_CAPACITY for a query longer than
 * max_batch_terms or
 * whose bitmap and id room exceed the whole pool; ABF_ERR_STATE once the
 * server is being destroyed. */
abf_status abf_server_submit(abf_server* server, const uint32_t* terms, uint32_t n_terms, uint64_t tag,
                             uint64_t arrival_ns, uint64_t* ticket);
/* Moves up to max_results finished queries into out, waiting up to
 * timeout_us for the first one. */
abf_status abf_server_poll(abf_server* server, abf_server_result* out, uint32_t max_results,
                           uint32_t timeout_us, uint32_t* n_out);
/* Frees a polled result (its device pointers become invalid). */
abf_status abf_server_release(abf_server* server, uint64_t ticket);
abf_status abf_server_get_stats(abf_server* server, abf_server_stats* out);
/* Fails the queries still waiting, waits for the batches in flight and
 * frees the pool (every result pointer becomes invalid). */
abf_status abf_server_destroy(abf_server* server);

/* Open-loop load: query i (terms[offsets[i] .. offsets[i+1])) is submitted
 * at start + arrival_ns[i] (ascending) by a generator thread, with that
 * time as its arrival; the calling thread polls and releases results as
 * they come. Per query: latency_ns (t_done - arrival; UINT64_MAX when
 * rejected or failed), and optionally queue_ns (launch - arrival), n_ids
 * and the path taken. Returns
 * when every query is done, or ABF_ERR_TIMEOUT after timeout_s. */
typedef struct abf_trace_stats {
    double seconds;              /* first arrival to last completion */
    uint64_t completed, rejected, failed;
} abf_trace_stats;
abf_status abf_server_run_trace(abf_server* server, const uint32_t* terms, const uint64_t* offsets,
                                uint32_t n_queries, const uint64_t* arrival_ns, double timeout_s,
                                uint64_t* h_latency_ns, uint64_t* h_queue_ns, uint64_t* h_n_ids,
                                uint8_t* h_paths,
                                abf_trace_stats* out);

/* ------------------------------------------------------------------ */
/* Misc                                                                */
/* ------------------------------------------------------------------ */
const char* abf_last_error_string(void);
const char* abf_status_string(abf_status s);
uint32_t abf_abi_version(void);
/* Number of kernel launches this library has enqueued since load. */
uint64_t abf_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* ADABOOL_H_ */
