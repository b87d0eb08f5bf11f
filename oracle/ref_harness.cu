// C wrapper around the reference's own single-query driver, compiled with
// nvcc for sm_100a from the reference sources where they lie (recipe:
// oracle/build_oracle.py). TEST AND BASELINE INFRASTRUCTURE ONLY.
//
// The driver file is included whole with its main() renamed, which brings
// in, unmodified, the reference's CPU path -- ComputeGroundTruth
// (test/adsfilter_q_all.cu:196-208) and CollectIdsFromBitmap
// (test/adsfilter_q_all.cu:108-119) -- and its GPU operator entry points
// ListUnion_dense / ListUnion_sparse (test/adsfilter_q_all.cu:26-105) with
// every kernel header they pull in (src/AdaBool/*.cu.h).
//
// The reference builds its index with a nested std::map
// (src/AdaBool/inverted_list.h:348-374), far too slow at 500M postings; the
// GPU entry points here take the arrays of the oracle's restatement of that
// builder (pinned array for array against the real one), load them through a
// subclass into the reference's own ivf_list, and let the reference compute
// its block metadata (ComputeKeyBlockSegments) and run its kernels.
#define main adsfilter_q_all_main
#include "adsfilter_q_all.cu"
#undef main

#include <atomic>
#include <thread>
#include <vector>

namespace {

struct RefIndex : public ivf_list<kKeyStep, kThreadNum> {
    // arrays per container type in the field order of abf_oracle.h
    void Load(const uint32_t* const* key_seg, const uint64_t* key_seg_len, const uint32_t* const* headers,
              const uint64_t* n_rec, const uint32_t* const* keys, const uint8_t* const* arrays,
              const uint64_t* arrays_len) {
        for (int t = 0; t < MAX_ARRAY_TYPE; ++t) {
            key_segments_[t].AllocFrom(key_seg[t], key_seg_len[t]);
            headers_[t].AllocFrom(headers[t], n_rec[t]);
            keys_[t].AllocFrom(keys[t], n_rec[t]);
            if (t != LIST_ARRAY1) arrays_[t].AllocFrom(arrays[t], arrays_len[t]);
        }
        ComputeKeyBlockSegments();
    }
};

struct CpuData {
    std::vector<std::pair<uint32_t, uint32_t>> kvs;
};

}  // namespace

extern "C" {

// ---------------- CPU path of the reference ----------------
void* refq_cpu_load(const uint32_t* terms, const uint32_t* ads, uint64_t nnz) {
    auto* d = new CpuData();
    d->kvs.resize(nnz);
    for (uint64_t i = 0; i < nnz; ++i) d->kvs[i] = {terms[i], ads[i]};
    return d;
}

void refq_cpu_free(void* h) { delete static_cast<CpuData*>(h); }

// ComputeGroundTruth for one query; ascending ids into out (cap), returns count
uint64_t refq_ground_truth(const void* h, const uint32_t* q, uint32_t nq, uint32_t* out, uint64_t cap) {
    const auto* d = static_cast<const CpuData*>(h);
    std::vector<uint32_t> query(q, q + nq);
    std::set<uint32_t> r = ComputeGroundTruth(d->kvs, query);
    uint64_t k = 0;
    for (uint32_t v : r) {
        if (k < cap) out[k] = v;
        ++k;
    }
    return k;
}

// ComputeGroundTruth over many queries on n_threads host threads
uint64_t refq_ground_truth_batch(const void* h, const uint64_t* q_off, const uint32_t* q_terms, uint32_t n_q,
                                 int n_threads, uint64_t* counts) {
    const auto* d = static_cast<const CpuData*>(h);
    std::atomic<uint32_t> next{0};
    auto body = [&] {
        for (;;) {
            uint32_t q = next.fetch_add(1);
            if (q >= n_q) break;
            std::vector<uint32_t> query(q_terms + q_off[q], q_terms + q_off[q + 1]);
            counts[q] = ComputeGroundTruth(d->kvs, query).size();
        }
    };
    std::vector<std::thread> th;
    for (int i = 0; i < (n_threads > 0 ? n_threads : 1); ++i) th.emplace_back(body);
    for (auto& t : th) t.join();
    uint64_t tot = 0;
    for (uint32_t q = 0; q < n_q; ++q) tot += counts[q];
    return tot;
}

uint64_t refq_collect_ids(const uint8_t* bitmap, uint64_t bytes, uint32_t* out, uint64_t cap) {
    std::vector<uint32_t> ids;
    CollectIdsFromBitmap(bitmap, bytes, ids);
    for (uint64_t k = 0; k < ids.size() && k < cap; ++k) out[k] = ids[k];
    return ids.size();
}

// ---------------- GPU path of the reference ----------------
void* refq_gpu_load(const uint32_t* const* key_seg, const uint64_t* key_seg_len, const uint32_t* const* headers,
                    const uint64_t* n_rec, const uint32_t* const* keys, const uint8_t* const* arrays,
                    const uint64_t* arrays_len) {
    auto* r = new RefIndex();
    r->Load(key_seg, key_seg_len, headers, n_rec, keys, arrays, arrays_len);
    return r;
}

void refq_gpu_free(void* h) { delete static_cast<RefIndex*>(h); }

// Prepare(len, bitmap) + ListUnion_dense into caller-zeroed d_res; the
// elapsed times (ms) of the prepare step (host clock) and of the kernels
// (CUDA events on the stream) go to *prep_ms and *kern_ms.
int refq_gpu_dense(void* h, const uint8_t* qbm, uint64_t len, uint32_t* d_res, void* stream, float* prep_ms,
                   float* kern_ms) {
    auto* r = static_cast<RefIndex*>(h);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto t0 = std::chrono::high_resolution_clock::now();
    auto w = r->Prepare(len, qbm);
    auto t1 = std::chrono::high_resolution_clock::now();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    ListUnion_dense(*w, d_res, s);
    cudaEventRecord(e1, s);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (prep_ms) *prep_ms = float(DurationMs(t0, t1));
    if (kern_ms) *kern_ms = ms;
    return err == cudaSuccess ? int(cudaGetLastError()) : int(err);
}

int refq_gpu_sparse(void* h, const uint32_t* keys, uint64_t n, uint32_t* d_res, void* stream, float* prep_ms,
                    float* kern_ms) {
    auto* r = static_cast<RefIndex*>(h);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<uint32_t> q(keys, keys + n);
    auto t0 = std::chrono::high_resolution_clock::now();
    auto w = r->Prepare(q);
    auto t1 = std::chrono::high_resolution_clock::now();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    ListUnion_sparse(*w, d_res, s);
    cudaEventRecord(e1, s);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (prep_ms) *prep_ms = float(DurationMs(t0, t1));
    if (kern_ms) *kern_ms = ms;
    return err == cudaSuccess ? int(cudaGetLastError()) : int(err);
}

// Batched bitmap-probe of 32 queries: PrepareBatch + RunArraysImpl<32>
// (src/AdaBool/inverted_list.h:564-574, src/AdaBool/inverted_list.cu.h:132-173),
// the path BatchListUnion_dense takes for batch_size 32
// (test/adsfilter_batch.cu:28-36). len is bytes per query bitmap (multiple of
// 16), res_len_u32 words per query result.
int refq_gpu_batch_dense32(void* h, const uint8_t* qbm, uint64_t len, uint32_t* d_res, uint32_t res_len_u32,
                           void* stream, float* prep_ms, float* kern_ms) {
    auto* r = static_cast<RefIndex*>(h);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto t0 = std::chrono::high_resolution_clock::now();
    auto w = r->PrepareBatch(32, len, qbm);
    auto t1 = std::chrono::high_resolution_clock::now();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    w->RunArraysImpl<32>(s, d_res, res_len_u32);
    cudaEventRecord(e1, s);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (prep_ms) *prep_ms = float(DurationMs(t0, t1));
    if (kern_ms) *kern_ms = ms;
    return err == cudaSuccess ? int(cudaGetLastError()) : int(err);
}

// Batched list-union: Prepare(flat keys) + the six RunSparseBatchListUnion*
// launches of BatchListUnion_sparse (test/adsfilter_batch.cu:39-79), restated
// here as glue because that driver file cannot be compiled alongside this one.
int refq_gpu_batch_sparse(void* h, const uint32_t* keys, const uint32_t* qidx, uint64_t n, uint32_t* d_res,
                          uint32_t res_len_bytes, void* stream, float* prep_ms, float* kern_ms) {
    auto* r = static_cast<RefIndex*>(h);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<uint32_t> q(keys, keys + n), qi(qidx, qidx + n);
    auto t0 = std::chrono::high_resolution_clock::now();
    auto w = r->Prepare(q);
    LenBuffer<INPUT, uint32_t> qidx_map;
    qidx_map.AllocFrom(qi);
    auto t1 = std::chrono::high_resolution_clock::now();
    const uint32_t rl = res_len_bytes / 4;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    const auto& T = w->tasks;
    RunSparseBatchListUnion1(T[LIST_ARRAY1].worker, s, d_res, qidx_map.d, rl, T[LIST_ARRAY1].indices_beg.d,
                             T[LIST_ARRAY1].d_value_headers, T[LIST_ARRAY1].d_value_arrays);
    RunSparseBatchListUnion<LIST_ARRAY4>(T[LIST_ARRAY4].worker, s, d_res, qidx_map.d, rl, T[LIST_ARRAY4].indices_beg.d,
                                         T[LIST_ARRAY4].d_value_headers, T[LIST_ARRAY4].d_value_arrays);
    RunSparseBatchListUnion<LIST_ARRAY8>(T[LIST_ARRAY8].worker, s, d_res, qidx_map.d, rl, T[LIST_ARRAY8].indices_beg.d,
                                         T[LIST_ARRAY8].d_value_headers, T[LIST_ARRAY8].d_value_arrays);
    RunSparseBatchListUnion<LIST_ARRAY16>(T[LIST_ARRAY16].worker, s, d_res, qidx_map.d, rl,
                                          T[LIST_ARRAY16].indices_beg.d, T[LIST_ARRAY16].d_value_headers,
                                          T[LIST_ARRAY16].d_value_arrays);
    RunSparseBatchListUnion<LIST_ARRAY32>(T[LIST_ARRAY32].worker, s, d_res, qidx_map.d, rl,
                                          T[LIST_ARRAY32].indices_beg.d, T[LIST_ARRAY32].d_value_headers,
                                          T[LIST_ARRAY32].d_value_arrays);
    RunSparseBatchListUnionBitset(T[LIST_BITSET].worker, s, d_res, qidx_map.d, rl, T[LIST_BITSET].indices_beg.d,
                                  T[LIST_BITSET].d_value_headers, T[LIST_BITSET].d_value_arrays);
    cudaEventRecord(e1, s);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (prep_ms) *prep_ms = float(DurationMs(t0, t1));
    if (kern_ms) *kern_ms = ms;
    return err == cudaSuccess ? int(cudaGetLastError()) : int(err);
}

}  // extern "C"
