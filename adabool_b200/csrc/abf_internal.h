// Internal structures of libadabool: the compressed list format, the index
// object, the workspace and the error plumbing shared by the host builder
// (abf_build.cpp), the generators (abf_gen.cpp), the kernels
// (abf_kernels.cu) and the C ABI (abf_capi.cu).
//
// List format (one array set for the whole index, all ids uint32):
//   - the postings of a term are cut into blocks of ABF_BLOCK_POSTINGS (128)
//     consecutive ids; every block but the last of a list is full;
//   - per block b: blk_first[b] = first id, blk_last[b] = last id,
//     blk_desc[b] = {payload offset in 16-byte units, bits | (count-1) << 8};
//   - the payload of a block is the bit-packed stream of its count-1 gaps
//     minus one: slot s (0 <= s < count-1) holds ids[s+1] - ids[s] - 1 in
//     `bits` bits at bit offset s*bits, little-endian within uint32 words;
//     bits = 0 means a run of consecutive ids and has no payload; the payload
//     is padded to a multiple of 16 bytes, so every block starts 16-byte
//     aligned and a warp stages it with one 16-byte load per lane;
//   - term_blk[t] .. term_blk[t+1] are the blocks of term t, term_len[t] its
//     length, blk_term[b] the term of block b (for the bitmap-probe scan).
// The reference stores ids as a 24-bit bucket plus 8-bit offsets in six
// fixed-width containers (src/AdaBool/inverted_list.h:16-26,390-470); this
// format replaces it and is not byte-compatible with it.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <atomic>

#include "../../include/adabool.h"

#ifndef __CUDACC__
struct alignas(16) abf_u4 { uint32_t x, y, z, w; };
struct alignas(8) abf_u2 { uint32_t x, y; };
#else
#include <cuda_runtime.h>
typedef uint4 abf_u4;
typedef uint2 abf_u2;
#endif

namespace abf {

constexpr uint32_t kBlock = ABF_BLOCK_POSTINGS;
constexpr uint32_t kMaxTileWords = 1024;

inline uint32_t desc_bits(uint32_t meta) { return meta & 63u; }
inline uint32_t desc_count(uint32_t meta) { return (meta >> 8) + 1u; }
inline uint32_t make_meta(uint32_t bits, uint32_t count) { return bits | ((count - 1u) << 8); }
// 16-byte units of payload for a block of `count` ids packed at `bits` bits.
inline uint32_t payload_units(uint32_t count, uint32_t bits) {
    uint64_t nbits = uint64_t(count - 1u) * bits;
    return uint32_t((nbits + 127u) / 128u);
}

// Host-side arrays of an index (the build output, the file payload and the
// source of every upload).
struct HostIndex {
    uint32_t n_terms = 0, n_ads = 0;
    uint64_t n_postings = 0;
    uint32_t max_list_len = 0;
    std::vector<uint32_t> term_blk;   // n_terms + 1
    std::vector<uint32_t> term_len;   // n_terms
    std::vector<uint32_t> blk_first;  // n_blocks
    std::vector<uint32_t> blk_last;   // n_blocks
    std::vector<uint32_t> blk_term;   // n_blocks
    std::vector<abf_u2> blk_desc;     // n_blocks
    std::vector<abf_u4> payload;      // payload units (+1 zero pad unit)
    uint64_t n_blocks() const { return blk_first.size(); }
};

// Tables derived from the lists at load time (not stored in the file):
//   - dense bitmaps: a list with len * dense_div >= n_ads also gets a
//     plain bitmap over all ads (dense_stride words, a multiple of 4); the
//     merge kernel ORs its tile slice instead of decoding the blocks;
//   - block directory: for long lists without a dense bitmap, dir[j] is
//     the first block whose last id is >= j * 2^kDirShift, so a tile finds
//     its blocks with three loads instead of two binary searches.
constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kDirShift = 13;      // directory granularity: 8192 ids = 256 words
constexpr uint32_t kDefaultDenseDiv = 128;
constexpr uint32_t kDirDiv = 512;       // lists with len * kDirDiv >= n_ads get a directory

struct DerivedHost {
    std::vector<uint32_t> term_dense;   // n_terms: dense bitmap index or kNone
    std::vector<uint32_t> dense;        // n_dense * dense_stride words
    uint64_t dense_stride = 0;
    uint32_t n_dense = 0;
    std::vector<uint32_t> term_dir;     // n_terms: offset into dir or kNone
    std::vector<uint32_t> dir;          // n_dir * dir_n absolute block indices
    uint32_t dir_n = 0;                 // entries per list: ceil(n_ads / 2^kDirShift) + 1
    uint32_t n_dir = 0;
};

// Device copies of the same arrays.
struct DeviceIndex {
    uint32_t* term_blk = nullptr;
    uint32_t* term_len = nullptr;
    uint32_t* blk_first = nullptr;
    uint32_t* blk_last = nullptr;
    uint32_t* blk_term = nullptr;
    abf_u2* blk_desc = nullptr;
    abf_u4* payload = nullptr;
    uint32_t* term_dense = nullptr;
    uint32_t* dense = nullptr;
    uint32_t* term_dir = nullptr;
    uint32_t* dir = nullptr;
    uint32_t* term_cbytes = nullptr;  // compressed bytes per term (planner feature)
    float* planner = nullptr;         // planner parameters (ABF_PLANNER_PARAMS) or null
    uint64_t bytes = 0;
};

// Read-only view passed to kernels by value.
struct IndexView {
    const abf_u4* payload;
    const uint32_t* blk_first;
    const uint32_t* blk_last;
    const abf_u2* blk_desc;
    const uint32_t* blk_term;
    const uint32_t* term_blk;
    const uint32_t* term_len;
    const uint32_t* term_dense;
    const uint32_t* dense;
    const uint32_t* term_dir;
    const uint32_t* dir;
    const uint32_t* term_cbytes;
    uint64_t dense_stride;
    uint32_t n_dense;
    uint32_t dir_n;
    uint32_t n_terms;
    uint32_t n_ads;
    uint64_t n_blocks;
};

}  // namespace abf

struct abf_workspace;

struct abf_index {
    abf::HostIndex host;          // emptied after upload unless kept
    abf::DerivedHost derived;     // dense bitmaps + directory (host copy until uploaded)
    uint32_t dense_div = abf::kDefaultDenseDiv;
    bool host_valid = false;      // host arrays hold the full index
    bool on_device = false;
    int device = -1;
    abf::DeviceIndex dev;
    // small host mirrors kept for planning and workers
    std::vector<uint32_t> h_term_blk;
    std::vector<uint32_t> h_term_len;
    std::vector<uint64_t> h_term_bytes;  // compressed bytes per term (payload + block metadata)
    bool prof_on = false;                 // kernel timing (abf_profile_enable)
    void* prof = nullptr;                 // event records, owned by abf_capi.cu
    uint64_t n_blocks = 0;
    uint64_t payload_units = 0;
    uint32_t n_terms = 0, n_ads = 0;
    uint64_t n_postings = 0;
    uint32_t max_list_len = 0;
    int sm_count = 148;
    abf_tuning tuning{};
    abf_workspace* own_ws = nullptr;  // for abf_query / abf_collect_ids
    void* h_stage = nullptr;          // pinned staging for abf_query terms
    size_t h_stage_bytes = 0;
    void* stage_event = nullptr;      // cudaEvent_t guarding the staging buffer
    // TMA descriptors of the dense bitmaps (2-D: words x bitmaps), encoded
    // on first use and again when the dense bitmaps or the tile width change
    alignas(64) unsigned char dense_tmap[256] = {};
    const void* dense_tmap_base = nullptr;
    uint32_t dense_tmap_rows = 0;
    uint32_t dense_tmap_gw = 0;       // tile words of the boxes (32 or 64)
};

namespace abf {

// thread-local error text; returns the status for `return fail(...)` use
abf_status fail(abf_status s, const std::string& msg);
void clear_error();
void count_launch(uint64_t n = 1);

// host builder entry (abf_build.cpp)
abf_status build_host(const uint64_t* offsets, const uint32_t* ads, uint32_t n_terms,
                      uint32_t n_ads, int n_threads, HostIndex* out);
abf_status save_host(const HostIndex& h, const char* path);
abf_status load_host(const char* path, HostIndex* h);
abf_status coo_to_csr(const uint32_t* terms, const uint32_t* ads, uint64_t nnz,
                      uint32_t n_terms, uint32_t n_ads, int n_threads,
                      std::vector<uint64_t>* offsets, std::vector<uint32_t>* csr_ads);
void decode_block_host(const HostIndex& h, uint64_t b, uint32_t* out);
int resolve_threads(int n);
// dense bitmaps and block directory of a host index (abf_build.cpp)
void derive_tables(const HostIndex& h, uint32_t dense_div, int n_threads, DerivedHost* out);

// device arrays of a workspace that the serving loop reads back after a
// batch (abf_capi.cu): the path each query ran on and the error flag
const uint8_t* ws_paths(const abf_workspace* w);
uint32_t* ws_err(abf_workspace* w);

}  // namespace abf
