// Kernel argument blocks and launchers of libadabool (sm_100a).
//
// Kernels (all integer, HBM/L2 bound):
//   plan_kernel        per query: resolve the path (given, the learned
//                      planner's inline, or the fixed rule), split lists into
//                      merged (long) and scattered (short), prefix the short
//                      lists' block counts, claim a bitmap-probe slot and
//                      write the probe query's term bitmap
//   queue_scan_kernel  exclusive scan of the per-query scattered block counts
//   tile_union_kernel  list-union, merge variant: one CTA owns a tile of one
//                      query's output bitmap in shared memory, decodes every
//                      block of the long lists that overlaps the tile, ORs
//                      with shared-memory atomics and writes the tile once
//   scatter_kernel     list-union, scatter variant: load-balanced warps decode
//                      the short lists' blocks and OR into the global bitmap
//                      with lane-combined atomicOr
//   probe_kernel       bitmap-probe: scans every block of the index, stages
//                      the probe queries' term-bitmap slices in shared memory
//                      with bulk async copies (TMA engine), tests each block's
//                      term and scatters hit blocks into their queries
//   compact_kernel     compaction: bitmap -> ascending uint32 ids in one pass
//                      (chunk popcounts, decoupled look-back prefix, id
//                      writes)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "abf_internal.h"

namespace abf {

constexpr uint32_t kNoHeavy = 0xffffffffu;   // heavy_min meaning "merge no list"
constexpr uint32_t kDenseOnly = 0xfffffffeu; // heavy_min meaning "merge only the dense-bitmap lists"
// warps per compaction CTA; a chunk (256 words per warp) fits one warp's id
// buffer, where the warp that prepares it stages it
constexpr uint32_t kCompactWarps = 4;
constexpr uint32_t kCompactChunkWords = kCompactWarps * 256;  // bitmap words per compaction work item
constexpr uint32_t kProbeGroup = 32;          // probe queries tested per pass

// device error codes (workspace flag)
constexpr uint32_t kErrScanTimeout = 1u;
constexpr uint32_t kErrTmaTimeout = 2u;
constexpr uint32_t kErrTermRange = 4u;

// Polls of a bounded device wait (look-back status word, mbarrier) before it
// gives up, sets its error bit and returns. A look-back poll sleeps ~64 ns,
// an mbarrier poll is one try_wait (which itself suspends for a
// hardware-defined interval), so the default allows well over a second.
constexpr uint32_t kDefaultSpinLimit = 1u << 22;

struct PlanArgs {
    const uint32_t* terms;
    const uint64_t* q_off;
    uint32_t n_q;
    const uint8_t* paths;     // per-query abf_path or null
    uint32_t path_uniform;    // abf_path when paths is null
    uint32_t hybrid_min;      // HYBRID merge threshold (postings)
    const float* planner;     // installed planner parameters (ABF_PLANNER_PARAMS) or null: with
                              // them, ABF_PATH_AUTO queries take the MLP's choice
    uint64_t n_postings;      // index postings (a planner feature)
    float probe_min_frac;     // fixed rule: probe when touched blocks / all blocks > this
    uint32_t fixed_hybrid_min;  // fixed rule otherwise: HYBRID when a list has >= this many
                                // postings (0: never), else UNION
    uint32_t* heavy_min;      // out: per query
    uint32_t* term_lpref;     // out: per term slot, exclusive prefix of scattered blocks
    uint64_t* q_light_cnt;    // out: per query scattered blocks
    uint32_t* probe_list;     // out: probe slot -> query
    uint32_t* n_probe;        // in/out: zeroed before launch
    uint32_t probe_cap;
    uint32_t* probe_bm;       // optional: probe slot s's term bitmap at probe_bm + s * probe_stride
    uint64_t probe_stride;    // words; written (zeroed, then the query's terms) by the query's CTA
    uint8_t* path_out;        // out (optional): resolved path per query
    uint64_t max_terms;       // term slots of the scratch arrays; queries past it get no work
    uint32_t* err;            // device error flag (optional)
    // optional: queries the merge kernel still has to visit when the dense
    // group kernel writes the dense-only ones (q_dmode != 1), compacted in
    // any order; n_tile_list is zeroed before launch
    uint32_t* tile_list;
    uint32_t* n_tile_list;
    int dense_in_tile;        // 1: dense-bitmap lists go to the merge kernel, 0: scattered too
    uint32_t* tile_cls;       // out: per term slot, what the merge kernel does with it
                              // (kNone: nothing, kDenseFlag | d: dense bitmap d, else the term)
    // optional per-query dense-bitmap lists (all four set, or q_dense16 null):
    // the query's distinct dense bitmap indices in ascending order, as 16-bit
    // values from q_dense16 + q_dstart[q] (16-byte aligned), padded to a
    // multiple of 8 with the index n_dense (an all-zero row for the TMA path)
    uint16_t* q_dense16;      // out: max_terms + 8 * n_q + 16 entries
    uint32_t* q_dstart;       // out: per query
    uint32_t* q_ndense;       // out: per query, distinct dense bitmaps
    uint32_t* q_dmode;        // out: per query, 1 if every list it merges has a dense bitmap,
                              // 2 if it also merges lists without one, 0 for probe / empty
};

constexpr uint32_t kDenseFlag = 0x80000000u;

struct QueueArgs {
    const uint64_t* q_light_cnt;
    uint64_t* q_light_pref;   // n_q + 1
    uint32_t n_q;
};

struct TileArgs {
    const uint32_t* tile_cls;  // per term slot, from the plan kernel
    const uint64_t* q_off;
    const uint32_t* heavy_min; // per query (null: heavy_all for every query)
    uint32_t heavy_all;
    uint32_t n_q;
    uint32_t n_tiles;
    uint32_t* out;
    uint64_t out_stride;      // words between query bitmaps
    uint64_t n_words;         // words of one bitmap
    int accumulate;           // 1: OR into the existing bitmap, 0: overwrite
    int vec_ok;               // out 16-byte aligned and out_stride % 4 == 0
    // optional (plan kernel): queries whose merged lists all have dense
    // bitmaps (q_dmode 1) take a barrier-free path that streams the OR of
    // their slices straight to the output, or are skipped when the dense
    // group kernel covers them; with the group kernel on (skip_dense_only),
    // q_dmode 2 queries start their tiles from its output and merge only
    // their lists without dense bitmaps
    const uint16_t* q_dense16;
    const uint32_t* q_dstart;
    const uint32_t* q_ndense;
    const uint32_t* q_dmode;
    int skip_dense_only;
    // with skip_dense_only: the plan kernel's list of the queries that are
    // not dense-only (the only ones this kernel visits) and its length
    const uint32_t* tile_list;
    const uint32_t* n_tile_list;
};

// dense group kernel: one pass per 32- or 64-word tile over all dense-only queries
constexpr uint32_t kGroupBoxRows = 256;   // dense bitmaps per TMA box
constexpr uint32_t kGroupMaxBoxes = 3;    // up to 767 dense bitmaps plus the zero row
constexpr uint32_t kGroupMaxQueries = 2048;
constexpr uint32_t kGroupSmemBytes = 226u * 1024u;  // dynamic shared memory of the group kernel

struct DenseGroupArgs {
    const uint16_t* q_dense16;
    const uint32_t* q_dstart;
    const uint32_t* q_ndense;
    const uint32_t* q_dmode;
    uint32_t n_q;              // <= kGroupMaxQueries
    uint32_t n_rows;           // n_dense + 1 (the last row reads as zeros)
    uint32_t list_cap;         // list entries (16-bit row word offsets) that fit in shared memory
    uint32_t stages;           // 2: double-buffered tile copies; 1: one stage, refilled after each tile
    uint32_t n_tiles;          // ceil(n_words / tile words)
    uint32_t* out;
    uint64_t out_stride;
    uint64_t n_words;
    uint32_t* err;
    uint32_t spin_limit;       // polls of an mbarrier wait before it gives up
    uint32_t* sat;             // optional, zeroed before launch: bit t of query q's sat_stride words
    uint32_t sat_stride;       //   is set when tile t of its bitmap came out all ones
};

struct ScatterArgs {
    const uint32_t* terms;
    const uint64_t* q_off;
    const uint32_t* term_lpref;
    const uint64_t* q_light_pref; // n_q + 1
    uint32_t n_q;
    const uint32_t* out_slot;  // query -> output bitmap index (null: identity)
    uint32_t* out;
    uint64_t out_stride;
    uint32_t blocks_per_warp;
    const uint32_t* sat;       // optional: the dense group kernel's saturated-tile bits
    uint32_t sat_stride;       //   (words per query); an OR into a word of such a tile
    uint32_t sat_shift;        //   is skipped; tile = word >> sat_shift
};

struct ProbeArgs {
    const uint32_t* qbm;       // probe term bitmaps, qbm_stride words apart
    uint64_t qbm_stride;
    uint32_t qbm_words;        // readable words per bitmap
    int staged_ok;             // qbm 16-byte aligned and stride % 4 == 0
    const uint32_t* d_n_probe; // device count, clamped to n_probe_host (null: n_probe_host)
    uint32_t n_probe_host;     // probe bitmaps available
    const uint32_t* out_slot;  // probe slot -> output bitmap index (null: identity)
    uint32_t* out;
    uint64_t out_stride;
    uint32_t chunk_blocks;     // multiple of 128
    uint32_t* err;
    uint32_t spin_limit;       // polls of an mbarrier wait before it gives up
};

// Compaction of n_q bitmaps into one packed id array. Work item i is chunk
// i % n_chunks of bitmap i / n_chunks; items are claimed in ascending order
// from a ticket counter, and each publishes its id count in status[i] so
// that later items find their output offset by looking back.
struct CompactArgs {
    const uint32_t* bm;
    uint64_t stride;           // words between bitmaps
    uint32_t n_q;
    uint64_t n_bits;           // ids >= n_bits are dropped
    uint32_t n_chunks;         // per bitmap
    uint64_t* status;          // n_q * n_chunks look-back words, zeroed before launch
    unsigned long long* ticket;  // item counter, zeroed before launch
    uint32_t* ids;
    uint64_t capacity;
    uint64_t* id_offsets;      // optional n_q + 1
    uint64_t* id_counts;       // optional n_q, accumulated (zeroed before launch)
    uint32_t* err;
    uint32_t spin_limit;       // polls of a look-back wait before it gives up
};

IndexView view_of(const abf_index* ix);
uint32_t compact_chunks(uint64_t n_bits);

cudaError_t launch_plan(const IndexView& v, const PlanArgs& a, cudaStream_t s);
// two 2-D TMA descriptors (2 x 128 bytes into out) of the dense bitmaps:
// gw-word (32 or 64) x 256-bitmap boxes, and one box for the remaining
// bitmaps plus the zero row; cudaErrorNotSupported when the driver has no
// encoder
cudaError_t encode_dense_tmap(const IndexView& v, uint32_t gw, void* out);
// list entries (16-bit row word offsets) the group kernel can stage in shared
// memory with gw-word tiles and `stages` stages (0: the stages do not fit)
uint32_t dense_group_list_cap(uint32_t n_rows, uint32_t n_q, uint32_t gw, uint32_t stages);
cudaError_t launch_dense_group(const void* tmaps, uint32_t gw, const DenseGroupArgs& a, int sm_count,
                               cudaStream_t s);
cudaError_t launch_queue_scan(const QueueArgs& a, cudaStream_t s);
cudaError_t launch_tile_union(const IndexView& v, const TileArgs& a, const abf_tuning& t, int sm_count,
                              cudaStream_t s);
cudaError_t launch_scatter(const IndexView& v, const ScatterArgs& a, const abf_tuning& t, int sm_count,
                           cudaStream_t s);
cudaError_t launch_probe(const IndexView& v, const ProbeArgs& a, const abf_tuning& t, int sm_count,
                         cudaStream_t s);
// planner (abf_planner.cu)
cudaError_t launch_planner(const IndexView& v, const float* params, const uint32_t* terms, const uint64_t* q_off,
                           uint32_t n_q, uint32_t hybrid_min, uint64_t n_postings, float* feat, float* pred,
                           uint8_t* paths, cudaStream_t s);
cudaError_t launch_mlp_forward(const float* p, const float* x, uint32_t n, float* y, cudaStream_t s);
cudaError_t launch_mlp_grad(const float* p, const float* x, const float* t, const float* mask, uint32_t n, float* g,
                            float* loss2, cudaStream_t s);
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, uint32_t step, float lr, float b1, float b2,
                        float eps, cudaStream_t s);

// clears status / ticket / id_counts on the stream, then one compaction launch
cudaError_t launch_compact(const CompactArgs& a, int sm_count, uint32_t ctas_per_sm, cudaStream_t s);

// Self-test of the bounded waits: one CTA arms an mbarrier for 16 bytes that
// no copy delivers, another looks back at a status word that no item
// publishes (status2[0], zeroed here); both run the same wait code as the
// path kernels with the given poll limit, give up, set kErrTmaTimeout /
// kErrScanTimeout in *err and return.
cudaError_t launch_wait_selftest(uint64_t* status2, uint32_t* err, uint32_t spin_limit, cudaStream_t s);

}  // namespace abf
