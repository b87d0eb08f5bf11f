// Thin C wrapper around the reference's own index builder, compiled with g++
// from the reference sources where they lie (recipe: oracle/build_oracle.py).
// TEST INFRASTRUCTURE ONLY: pins the oracle's restatement of the mixed
// container format (oracle/abf_oracle.c) array for array.
//
// Without __CUDACC__ the reference's LenBuffer keeps host memory only
// (src/AdaBool/len_buffer.h:222-226), so BuildFrom runs on a machine
// without a GPU. The reference headers miss two standard includes; the
// recipe passes them with -include.
#include "inverted_list.h"

#include <cstdint>
#include <utility>
#include <vector>

namespace {
// exposes the protected arrays of ivf_list
struct RefBuilt : public ivf_list<256, 64> {
    int get(int t, int f, const void** p, uint64_t* len) const {
        if (t < 0 || t >= MAX_ARRAY_TYPE) return -1;
        switch (f) {
            case 0: *p = key_segments_[t].h; *len = key_segments_[t].len; return 0;
            case 1: *p = headers_[t].h; *len = headers_[t].len; return 0;
            case 2: *p = keys_[t].h; *len = keys_[t].len; return 0;
            case 3: *p = arrays_[t].h; *len = arrays_[t].len; return 0;
            case 4: *p = key_array_metas_[t].key_pos_segments.h; *len = key_array_metas_[t].key_pos_segments.len; return 0;
            case 5: *p = key_array_metas_[t].key_block_segments.h; *len = key_array_metas_[t].key_block_segments.len; return 0;
            case 6: *p = key_array_metas_[t].key_buffers.h; *len = key_array_metas_[t].key_buffers.len; return 0;
            default: return -1;
        }
    }
};
}  // namespace

extern "C" {

void* refb_build(const uint32_t* terms, const uint32_t* ads, uint64_t nnz) {
    std::vector<std::pair<uint32_t, uint32_t>> kv(nnz);
    for (uint64_t i = 0; i < nnz; ++i) kv[i] = {terms[i], ads[i]};
    auto* r = new RefBuilt();
    r->BuildFrom(kv);
    return r;
}

int refb_array(const void* h, int type, int field, const void** p, uint64_t* len) {
    return static_cast<const RefBuilt*>(h)->get(type, field, p, len);
}

void refb_free(void* h) { delete static_cast<RefBuilt*>(h); }
}
