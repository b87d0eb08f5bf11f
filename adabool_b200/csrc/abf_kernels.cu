// Kernels of libadabool for sm_100a. See abf_kernels.cuh for the overview
// and abf_internal.h for the list format they decode.
//
// Reference counterparts (yxr620/AdaBool):
//   scatter_kernel / tile_union_kernel  <- ListUnionKernel{1,,Bitset} and
//       SparseBatchListUnionKernel{1,,Bitset}
//       (src/AdaBool/load_balance_transformer.cu.h:16-91,138-220) with the
//       container decoders (src/AdaBool/inverted_list.cu.h:61-130)
//   probe_kernel  <- KeyBPTransformKernel{1,,Bitset} and
//       KeyBatchBPTransformKernel_Expanded{1,,Bitset}
//       (src/AdaBool/key_transformer.cu.h:11-331,
//        src/AdaBool/key_batch_transformer.cu.h:11-524)
//   count/scan/write  <- the host loop CollectIdsFromBitmap
//       (test/adsfilter_batch.cu:82-97)
#include "abf_kernels.cuh"
#include "abf_planner_dev.cuh"

#include <cuda.h>
#include <cstring>

#include <algorithm>
#include <atomic>

namespace abf {

namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kProbeSmemWords = 8192;  // staged term-bitmap words per CTA
// look-back status word: flag in the top two bits, count below
constexpr uint64_t kFlagAgg = 1ull << 62;   // the item's own id count is known
constexpr uint64_t kFlagIncl = 2ull << 62;  // the ids of the item and all before it
constexpr uint64_t kValMask = (1ull << 62) - 1;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t warp_id() { return threadIdx.x >> 5; }

// ---------------------------------------------------------------------------
// block decode: one warp, one block of up to 128 ids
// ---------------------------------------------------------------------------
// Lane j returns the ids of positions 4j..4j+3 of the block (ascending across
// the warp); position i is valid when i < cnt. The payload is staged in the
// warp's 512-byte shared buffer with one 16-byte load per lane; each lane
// extracts its four gaps with a funnel shift, sums them, and a shuffle scan
// over the lanes turns the gaps into ids.
// A block's descriptor and this lane's 16 bytes of its payload, loaded
// ahead of the decode so the loads of the next block overlap the work on
// the current one.
struct Fetched {
    uint4 pay;
    uint32_t first, meta;
};

__device__ __forceinline__ Fetched fetch_block(const IndexView& ix, uint32_t b) {
    Fetched r;
    const uint2 d = __ldg(ix.blk_desc + b);
    r.first = __ldg(ix.blk_first + b);
    r.meta = d.y;
    const uint32_t bits = d.y & 63u, cnt = (d.y >> 8) + 1u;
    const uint32_t units = ((cnt - 1u) * bits + 127u) >> 7;
    r.pay = lane_id() < units ? __ldg(ix.payload + d.x + lane_id()) : make_uint4(0u, 0u, 0u, 0u);
    return r;
}

__device__ __forceinline__ void decode_fetched(const Fetched& fb, uint4* stage, uint32_t (&id)[4], uint32_t& cnt) {
    const uint32_t lane = lane_id();
    const uint32_t first = fb.first;
    const uint32_t bits = fb.meta & 63u;
    cnt = (fb.meta >> 8) + 1u;
    __syncwarp();
    stage[lane] = fb.pay;
    __syncwarp();
    const uint32_t* w = reinterpret_cast<const uint32_t*>(stage);
    const uint32_t mask = bits >= 32u ? kFull : ((1u << bits) - 1u);
    uint32_t p[4];
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t i = lane * 4u + k;
        uint32_t g = 0;
        if (i >= 1u && i < cnt) {
            uint32_t v = 0;
            if (bits) {
                const uint32_t pos = (i - 1u) * bits;
                const uint32_t wi = pos >> 5;
                v = __funnelshift_r(w[wi], w[wi + 1], pos & 31u) & mask;
            }
            g = v + 1u;
        }
        run += g;
        p[k] = run;
    }
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane >= uint32_t(o)) incl += y;
    }
    const uint32_t base = first + (incl - run);
#pragma unroll
    for (int k = 0; k < 4; ++k) id[k] = base + p[k];
}

__device__ __forceinline__ void decode_block(const IndexView& ix, uint32_t b, uint4* stage, uint32_t (&id)[4],
                                             uint32_t& cnt) {
    decode_fetched(fetch_block(ix, b), stage, id, cnt);
}

// OR the decoded ids that fall in [lo, lo + span) into a shared-memory tile.
// A lane's ids are ascending, so runs in one word are combined before the
// atomic.
__device__ __forceinline__ void or_tile(uint32_t* tile, uint32_t lo, uint32_t span, const uint32_t (&id)[4],
                                        uint32_t cnt) {
    const uint32_t lane = lane_id();
    uint32_t cur = kFull, m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t i = lane * 4u + k;
        const uint32_t rel = id[k] - lo;
        if (i < cnt && rel < span) {
            const uint32_t wd = rel >> 5, bit = 1u << (rel & 31u);
            if (wd != cur) {
                if (cur != kFull) atomicOr(tile + cur, m);
                cur = wd;
                m = bit;
            } else {
                m |= bit;
            }
        }
    }
    if (cur != kFull) atomicOr(tile + cur, m);
}

// OR decoded ids (< n_ads) into a global bitmap, same lane-local combining.
// true when word wd lies in a tile whose bits are all set already
__device__ __forceinline__ bool in_full_tile(const uint32_t* sat, uint32_t sat_shift, uint32_t wd) {
    const uint32_t t = wd >> sat_shift;
    return (__ldg(sat + (t >> 5)) >> (t & 31u)) & 1u;
}

// true when every tile that ids [lo, hi) can touch is marked all ones
// (tile = word >> sat_shift): the whole block can be skipped, decode
// included. Ranges over more than 32 words of marks are not checked.
__device__ __forceinline__ bool range_saturated(const uint32_t* sat, uint32_t sat_shift, uint32_t lo, uint32_t hi) {
    const uint32_t t0 = (lo >> 5) >> sat_shift, t1 = ((hi - 1u) >> 5) >> sat_shift;
    const uint32_t w0 = t0 >> 5, nw = (t1 >> 5) - w0 + 1u;
    if (nw > 32u) return false;  // warp-uniform
    const uint32_t lane = lane_id();
    bool ok = true;
    if (lane < nw) {
        uint32_t m = ~0u;
        if (lane == 0) m &= ~0u << (t0 & 31u);
        if (lane + 1u == nw) m &= ~0u >> (31u - (t1 & 31u));
        ok = (__ldg(sat + w0 + lane) & m) == m;
    }
    return __all_sync(kFull, ok);
}

// OR of this lane's four ids into the bitmap, one atomic per distinct word;
// with sat (the dense group kernel's saturated-tile bits of this bitmap),
// words inside an all-ones tile are skipped: the OR cannot change them
__device__ __forceinline__ void or_global(uint32_t* bm, uint32_t n_ads, const uint32_t (&id)[4], uint32_t cnt,
                                          const uint32_t* sat = nullptr, uint32_t sat_shift = 0) {
    const uint32_t lane = lane_id();
    uint32_t cur = kFull, m = 0;
    auto flush = [&]() {
        if (!sat || !in_full_tile(sat, sat_shift, cur)) atomicOr(bm + cur, m);
    };
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t i = lane * 4u + k;
        if (i < cnt && id[k] < n_ads) {
            const uint32_t wd = id[k] >> 5, bit = 1u << (id[k] & 31u);
            if (wd != cur) {
                if (cur != kFull) flush();
                cur = wd;
                m = bit;
            } else {
                m |= bit;
            }
        }
    }
    if (cur != kFull) flush();
}

template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    constexpr int NWARP = NT / 32;
    const uint32_t lane = lane_id(), warp = warp_id();
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= uint32_t(o)) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < uint32_t(NWARP) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, w, o);
            if (lane >= uint32_t(o)) w += y;
        }
        if (lane < uint32_t(NWARP)) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t wex = warp ? s_warp[warp - 1] : 0u;
    *total = s_warp[NWARP - 1];
    __syncthreads();
    return wex + x - v;
}

template <int NT>
__device__ __forceinline__ uint64_t block_sum_u64(uint64_t v, unsigned long long* s) {
    const uint32_t lane = lane_id(), warp = warp_id();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    if (lane == 0) s[warp] = v;
    __syncthreads();
    uint64_t t = 0;
    for (int i = 0; i < NT / 32; ++i) t += s[i];
    __syncthreads();
    return t;
}

// first index in [a, b) with arr[index] >= key (arr ascending)
__device__ __forceinline__ uint32_t lower_bound_g(const uint32_t* arr, uint32_t a, uint32_t b, uint32_t key) {
    while (a < b) {
        const uint32_t m = (a + b) >> 1;
        if (__ldg(arr + m) < key) a = m + 1; else b = m;
    }
    return a;
}

// ---------------------------------------------------------------------------
// mbarrier + bulk async copy (TMA engine, 1-D form)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of `bar` with the given parity; false after `limit`
// polls without it completing.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t spins = 0; !mbar_try_wait(bar, parity);)
        if (++spins > limit) return false;
    return true;
}

// ---------------------------------------------------------------------------
// planning
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 4) plan_kernel(IndexView ix, PlanArgs a) {
    __shared__ uint32_t s_warp[32];
    __shared__ unsigned long long s_red[8];
    __shared__ uint32_t s_path, s_max, s_slot;
    __shared__ uint32_t s_mask[2048];  // the query's dense bitmaps (n_dense <= 65535)
    __shared__ plan_dev::PlannerSmem s_pl;
    static_assert(plan_dev::kFeatThreads == 256, "the planner code runs with the plan kernel's 256 threads");
    const uint32_t tid = threadIdx.x;
    for (uint32_t q = blockIdx.x; q < a.n_q; q += gridDim.x) {
        uint64_t qb = a.q_off[q], qe = a.q_off[q + 1];
        if (qe < qb || qe > a.max_terms) {
            // offsets outside the scratch arrays: the query gets no work
            if (tid == 0 && a.err) atomicOr(a.err, kErrTermRange);
            qe = qb = 0;
        }
        uint32_t path = a.paths ? a.paths[q] : a.path_uniform;
        if (path == ABF_PATH_AUTO && a.planner) {
            // learned planner: features + MLP of this query, inline
            path = plan_dev::planner_path(ix, a.planner, a.terms, a.q_off, q,
                                          plan_dev::FeatCtx{a.hybrid_min, a.n_postings, a.n_q}, s_pl);
        } else if (path == ABF_PATH_AUTO) {
            // fixed rule: probe when the query's lists cover more than
            // probe_min_frac of all blocks; else HYBRID when one of its lists
            // has at least fixed_hybrid_min postings; else list-union
            uint64_t nb = 0;
            uint32_t mx = 0;
            for (uint64_t i = qb + tid; i < qe; i += 256) {
                const uint32_t t = a.terms[i];
                if (t < ix.n_terms) {
                    nb += __ldg(ix.term_blk + t + 1) - __ldg(ix.term_blk + t);
                    mx = max(mx, __ldg(ix.term_len + t));
                }
            }
            if (tid == 0) s_max = 0;
            nb = block_sum_u64<256>(nb, s_red);  // its barriers also order the s_max reset
            mx = __reduce_max_sync(kFull, mx);
            if (lane_id() == 0 && mx) atomicMax(&s_max, mx);
            __syncthreads();
            mx = s_max;
            path = (double(nb) > double(a.probe_min_frac) * double(ix.n_blocks)) ? ABF_PATH_PROBE
                   : (a.fixed_hybrid_min && mx >= a.fixed_hybrid_min) ? ABF_PATH_HYBRID
                                                                      : ABF_PATH_UNION;
        }
        if (tid == 0) {
            s_slot = kNone;
            if (path == ABF_PATH_PROBE) {
                const uint32_t slot = atomicAdd(a.n_probe, 1u);
                if (slot < a.probe_cap) {
                    a.probe_list[slot] = q;
                    s_slot = slot;
                } else {
                    path = ABF_PATH_UNION;  // no probe slot left: same result by list-union
                }
            }
            s_path = path;
        }
        __syncthreads();
        path = s_path;
        const bool probe = path == ABF_PATH_PROBE;
        if (probe && a.probe_bm) {
            // the probe slot's term bitmap: zeroed, then this query's terms
            uint32_t* bm = a.probe_bm + uint64_t(s_slot) * a.probe_stride;
            for (uint64_t w = tid; w < a.probe_stride; w += 256) bm[w] = 0u;
            __syncthreads();
            for (uint64_t i = qb + tid; i < qe; i += 256) {
                const uint32_t t = a.terms[i];
                if (t < ix.n_terms) atomicOr(bm + (t >> 5), 1u << (t & 31u));
            }
        }
        // merge threshold: TILE merges every list, HYBRID the long ones,
        // UNION only those with a dense bitmap, PROBE none
        const uint32_t hm = path == ABF_PATH_TILE ? 0u
                            : path == ABF_PATH_HYBRID ? a.hybrid_min
                            : probe ? kNoHeavy : kDenseOnly;
        const bool want_d = a.q_dense16 != nullptr;
        const uint32_t mw = (ix.n_dense + 31u) / 32u;
        if (want_d) {
            for (uint32_t i = tid; i < mw; i += 256) s_mask[i] = 0u;
            __syncthreads();
        }
        uint32_t carry = 0, nmerge = 0;
        for (uint64_t c0 = qb; c0 < qe; c0 += 256) {
            const uint64_t i = c0 + tid;
            uint32_t cnt = 0, cls = kNone;
            if (i < qe && !probe) {
                const uint32_t t = a.terms[i];
                if (t < ix.n_terms) {
                    const uint32_t d = a.dense_in_tile ? __ldg(ix.term_dense + t) : kNone;
                    const uint32_t len = __ldg(ix.term_len + t);
                    if (d != kNone) cls = kDenseFlag | d;
                    else if (len >= hm) cls = t;
                    else cnt = __ldg(ix.term_blk + t + 1) - __ldg(ix.term_blk + t);
                }
            }
            if (i < qe && a.tile_cls) a.tile_cls[i] = cls;
            uint32_t tot;
            const uint32_t ex = block_excl_scan<256>(cnt, s_warp, &tot);
            if (i < qe) a.term_lpref[i] = carry + ex;
            carry += tot;
            if (want_d && cls != kNone) {
                if (cls & kDenseFlag) {
                    const uint32_t d = cls & ~kDenseFlag;
                    atomicOr(&s_mask[d >> 5], 1u << (d & 31u));
                } else {
                    ++nmerge;
                }
            }
        }
        if (want_d) {
            // the query's distinct dense bitmaps in ascending order: each
            // thread expands a contiguous run of mask words at its prefix
            const uint32_t any_merge = __syncthreads_or(nmerge);
            const uint32_t per = (mw + 255u) / 256u;
            const uint32_t w0 = tid * per < mw ? tid * per : mw;
            const uint32_t w1 = w0 + per < mw ? w0 + per : mw;
            uint32_t c = 0;
            for (uint32_t w = w0; w < w1; ++w) c += __popc(s_mask[w]);
            uint32_t nd;
            uint32_t o = block_excl_scan<256>(c, s_warp, &nd);
            const uint32_t start = uint32_t((qb + 8ull * q + 7ull) & ~7ull);
            uint16_t* dst = a.q_dense16 + start;
            for (uint32_t w = w0; w < w1; ++w) {
                uint32_t m = s_mask[w];
                while (m) {
                    dst[o++] = uint16_t(w * 32u + uint32_t(__ffs(m)) - 1u);
                    m &= m - 1u;
                }
            }
            for (uint32_t i = nd + tid; i < ((nd + 7u) & ~7u); i += 256) dst[i] = uint16_t(ix.n_dense);
            if (tid == 0) {
                a.q_dstart[q] = start;
                a.q_ndense[q] = nd;
                // 1: every list it merges has a dense bitmap; 2: it also merges
                // lists without one; 0: probe or empty (no dense merge at all)
                const uint32_t dmode = (!probe && qe > qb) ? (any_merge ? 2u : 1u) : 0u;
                a.q_dmode[q] = dmode;
                if (a.tile_list && dmode != 1u) a.tile_list[atomicAdd(a.n_tile_list, 1u)] = q;
            }
        }
        if (tid == 0) {
            a.heavy_min[q] = probe ? kNoHeavy : hm;
            a.q_light_cnt[q] = carry;
            if (a.path_out) a.path_out[q] = uint8_t(path);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) queue_scan_kernel(QueueArgs a) {
    __shared__ unsigned long long s_warp[32];
    __shared__ unsigned long long s_carry;
    const uint32_t tid = threadIdx.x, lane = lane_id(), warp = warp_id();
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < a.n_q; c0 += 1024) {
        const uint32_t i = c0 + tid;
        const uint64_t v = i < a.n_q ? a.q_light_cnt[i] : 0ull;
        uint64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= uint32_t(o)) x += y;
        }
        if (lane == 31) s_warp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint64_t w = s_warp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(kFull, w, o);
                if (lane >= uint32_t(o)) w += y;
            }
            s_warp[lane] = w;
        }
        __syncthreads();
        const uint64_t base = s_carry + (warp ? s_warp[warp - 1] : 0ull);
        if (i < a.n_q) a.q_light_pref[i] = base + x - v;
        __syncthreads();
        if (tid == 0) s_carry += s_warp[31];
        __syncthreads();
    }
    if (tid == 0) a.q_light_pref[a.n_q] = s_carry;
}

// ---------------------------------------------------------------------------
// list-union, merge variant
// ---------------------------------------------------------------------------
// Blocks [lo, lo + cnt) of a list that overlap the ids [lo_id, hi_id):
// three loads from the list's directory when it has one, else two binary
// searches over the block bounds. dj0/dj1 are the directory rows of lo_id
// and of the unclipped tile end.
__device__ __forceinline__ void tile_block_range(const IndexView& ix, uint32_t term, uint32_t lo_id, uint32_t hi_id,
                                                 uint32_t dj0, uint32_t dj1, uint32_t& lo, uint32_t& cnt) {
    const uint32_t b0 = __ldg(ix.term_blk + term), b1 = __ldg(ix.term_blk + term + 1);
    const uint32_t dofs = __ldg(ix.term_dir + term);
    uint32_t hi;
    if (dofs != kNone) {
        lo = __ldg(ix.dir + dofs + dj0);
        hi = __ldg(ix.dir + dofs + dj1);  // first block ending at or after the tile end
        if (hi < b1 && __ldg(ix.blk_first + hi) < hi_id) ++hi;  // it straddles the tile end
    } else {
        lo = lower_bound_g(ix.blk_last, b0, b1, lo_id);
        hi = lower_bound_g(ix.blk_first, lo, b1, hi_id);
    }
    cnt = hi > lo ? hi - lo : 0u;
}

// slot s of the chunk's prefix array with s_pref[s] <= f < s_pref[s+1]
template <int NT>
__device__ __forceinline__ uint32_t find_slot(const uint32_t* s_pref, uint32_t f) {
    uint32_t a0 = 0, a1 = NT;
    while (a1 - a0 > 1) {
        const uint32_t m = (a0 + a1) >> 1;
        if (s_pref[m] <= f) a0 = m; else a1 = m;
    }
    return a0;
}

// One tile of a query whose merged lists all have dense bitmaps: the OR of
// the nd slices [t*W, t*W + nw) of the bitmaps listed in dl, written to dst.
template <int W, int NT>
__device__ __forceinline__ void dense_only_tile(const IndexView& ix, const uint16_t* dl, uint32_t nd, uint32_t t,
                                                uint32_t* dst, uint32_t nw, bool vec_ok) {
    constexpr uint32_t KT = 8;
    const uint32_t tid = threadIdx.x;
    const uint64_t tw = uint64_t(t) * W;
    if (vec_ok) {
        const uint4* base = reinterpret_cast<const uint4*>(ix.dense + tw);
        const uint64_t st4 = ix.dense_stride / 4;
        uint4* d4 = reinterpret_cast<uint4*>(dst);
        const uint32_t n4 = nw / 4u;
        for (uint32_t j = tid; j < n4; j += NT) {
            uint4 acc = make_uint4(0u, 0u, 0u, 0u);
            uint32_t k = 0;
            for (; k + KT <= nd; k += KT) {
                uint4 x[KT];
#pragma unroll
                for (uint32_t e = 0; e < KT; ++e) x[e] = __ldg(base + uint64_t(__ldg(dl + k + e)) * st4 + j);
#pragma unroll
                for (uint32_t e = 0; e < KT; ++e) {
                    acc.x |= x[e].x; acc.y |= x[e].y; acc.z |= x[e].z; acc.w |= x[e].w;
                }
                // lists come longest first: a saturated slice reads no more rows
                if ((acc.x & acc.y & acc.z & acc.w) == ~0u) break;
            }
            if ((acc.x & acc.y & acc.z & acc.w) == ~0u) k = nd;
            for (; k < nd; ++k) {
                const uint4 x = __ldg(base + uint64_t(__ldg(dl + k)) * st4 + j);
                acc.x |= x.x; acc.y |= x.y; acc.z |= x.z; acc.w |= x.w;
            }
            d4[j] = acc;
        }
        for (uint32_t i = n4 * 4u + tid; i < nw; i += NT) {
            uint32_t acc = 0;
            for (uint32_t k = 0; k < nd; ++k) acc |= __ldg(ix.dense + uint64_t(__ldg(dl + k)) * ix.dense_stride + tw + i);
            dst[i] = acc;
        }
    } else {
        for (uint32_t i = tid; i < nw; i += NT) {
            uint32_t acc = 0;
            for (uint32_t k = 0; k < nd; ++k) acc |= __ldg(ix.dense + uint64_t(__ldg(dl + k)) * ix.dense_stride + tw + i);
            dst[i] = acc;
        }
    }
}

template <int W, int NW>
__global__ void __launch_bounds__(NW * 32) tile_union_kernel(IndexView ix, TileArgs a) {
    constexpr int NT = NW * 32;
    constexpr uint32_t SPAN = uint32_t(W) * 32u;
    extern __shared__ __align__(16) uint32_t tile[];  // W words, dynamic (up to 64 KB)
    __shared__ __align__(16) uint4 stage[NW][32];
    __shared__ uint32_t s_lo[NT];
    __shared__ uint32_t s_pref[NT + 1];
    __shared__ uint32_t s_dense[NT];
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_ndense;
    const uint32_t tid = threadIdx.x, warp = warp_id();
    // with the dense group kernel writing the dense-only queries, only the
    // plan kernel's list of the other queries is visited (often none)
    const bool listed = a.skip_dense_only && a.tile_list;
    const uint32_t n_q = listed ? *a.n_tile_list : a.n_q;
    const uint64_t items = uint64_t(n_q) * a.n_tiles;
    uint4* tile4 = reinterpret_cast<uint4*>(tile);
    for (uint64_t item = blockIdx.x; item < items; item += gridDim.x) {
        // tile-major order: the CTAs resident together work on one region of
        // the ad space for many queries, so the blocks and dense slices of
        // lists those queries share are read from L2
        const uint32_t t = uint32_t(item / n_q);
        const uint32_t qi = uint32_t(item - uint64_t(t) * n_q);
        const uint32_t q = listed ? a.tile_list[qi] : qi;
        const uint32_t lo_id = t * SPAN;
        const uint32_t hi_id = (uint64_t(lo_id) + SPAN > ix.n_ads) ? ix.n_ads : lo_id + SPAN;
        const uint32_t dj0 = lo_id >> kDirShift;
        uint32_t dj1 = uint32_t((uint64_t(lo_id) + SPAN) >> kDirShift);
        if (dj1 > ix.dir_n - 1) dj1 = ix.dir_n - 1;
        const uint32_t hm = a.heavy_min ? a.heavy_min[q] : a.heavy_all;
        const uint64_t qb = a.q_off[q], qe = a.q_off[q + 1];
        uint32_t* dst = a.out + uint64_t(q) * a.out_stride + uint64_t(t) * W;
        const uint64_t left = a.n_words - uint64_t(t) * W;
        const uint32_t nw = left < uint64_t(W) ? uint32_t(left) : uint32_t(W);
        if (hm == kNoHeavy || qb == qe) {  // nothing to merge: leave or zero the tile
            if (!a.accumulate)
                for (uint32_t i = tid; i < nw; i += NT) dst[i] = 0u;
            continue;
        }
        const uint32_t dmode = a.q_dense16 ? a.q_dmode[q] : 0u;
        if (a.q_dense16 && !a.accumulate && dmode == 1u) {
            // every merged list has a dense bitmap: the dense group kernel
            // writes this tile, or each thread ORs its 16-byte slots over the
            // query's dense slices, KT loads in flight, and stores the
            // result; no shared tile, no barrier
            if (!a.skip_dense_only)
                dense_only_tile<W, NT>(ix, a.q_dense16 + a.q_dstart[q], a.q_ndense[q], t, dst, nw, a.vec_ok != 0);
            continue;
        }
        // with the dense group kernel on, a query that also merges lists
        // without dense bitmaps already has its dense lists in the output:
        // the tile starts from it and adds only the others
        const bool on_group = a.skip_dense_only && dmode == 2u && !a.accumulate;
        for (uint32_t i = tid; i < uint32_t(W); i += NT) tile[i] = ((a.accumulate || on_group) && i < nw) ? dst[i] : 0u;
        if (tid == 0) s_ndense = 0;
        __syncthreads();
        for (uint64_t c0 = qb; c0 < qe; c0 += NT) {
            const uint64_t i = c0 + tid;
            uint32_t lo = 0, cnt = 0;
            const uint32_t cls = i < qe ? __ldg(a.tile_cls + i) : kNone;
            if (cls != kNone) {
                if (cls & kDenseFlag) {
                    if (!on_group) s_dense[atomicAdd(&s_ndense, 1u)] = cls & ~kDenseFlag;
                } else {
                    tile_block_range(ix, cls, lo_id, hi_id, dj0, dj1, lo, cnt);
                }
            }
            uint32_t total;
            const uint32_t ex = block_excl_scan<NT>(cnt, s_warp, &total);
            s_lo[tid] = lo;
            s_pref[tid] = ex;
            if (tid == NT - 1) s_pref[NT] = ex + cnt;
            __syncthreads();
            // dense lists: OR their slice of this tile, 16 bytes per thread and
            // slot, four lists' loads in flight at once; finished before any
            // decode warp starts its shared atomics
            const uint32_t nd = s_ndense;
            if (nd) {
                // each thread keeps VG of its 16-byte slots in registers and
                // issues VG x KT independent loads per step (KT lists at once)
                constexpr int V = (W / 4 + NT - 1) / NT;
                constexpr int VG = V < 4 ? V : 4;
                constexpr int KT = VG >= 4 ? 2 : (VG == 2 ? 4 : 8);
                const uint4* base = reinterpret_cast<const uint4*>(ix.dense + uint64_t(t) * W);
                const uint64_t st4 = ix.dense_stride / 4;
                for (int vg = 0; vg < V; vg += VG) {
                    uint4 acc[VG];
#pragma unroll
                    for (int v = 0; v < VG; ++v) {
                        const uint32_t j = tid + uint32_t(vg + v) * NT;
                        acc[v] = j * 4u < nw ? tile4[j] : make_uint4(0u, 0u, 0u, 0u);
                    }
                    for (uint32_t k = 0; k < nd; k += KT) {
                        const uint4* src[KT];
#pragma unroll
                        for (int e = 0; e < KT; ++e)
                            src[e] = base + uint64_t(s_dense[k + e < nd ? k + e : k]) * st4;
#pragma unroll
                        for (int v = 0; v < VG; ++v) {
                            const uint32_t j = tid + uint32_t(vg + v) * NT;
                            if (j * 4u < nw) {
                                uint4 x[KT];
#pragma unroll
                                for (int e = 0; e < KT; ++e) x[e] = __ldg(src[e] + j);
#pragma unroll
                                for (int e = 0; e < KT; ++e) {
                                    acc[v].x |= x[e].x; acc[v].y |= x[e].y; acc[v].z |= x[e].z; acc[v].w |= x[e].w;
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int v = 0; v < VG; ++v) {
                        const uint32_t j = tid + uint32_t(vg + v) * NT;
                        if (j * 4u < nw) tile4[j] = acc[v];
                    }
                }
            }
            __syncthreads();
            // decode the blocks: warp w takes a contiguous share of the flat
            // block range, finds its first (slot, block) once and walks on,
            // keeping the next block's loads in flight
            const uint32_t per = (total + NW - 1) / NW;
            uint32_t f = warp * per;
            const uint32_t fend = f + per < total ? f + per : total;
            if (f < fend) {
                uint32_t s = find_slot<NT>(s_pref, f);
                uint32_t j = f - s_pref[s];
                Fetched nxt = fetch_block(ix, s_lo[s] + j);
                while (f < fend) {
                    const Fetched cur = nxt;
                    if (++f < fend) {
                        if (++j == s_pref[s + 1] - s_pref[s]) {  // next list with blocks in this tile
                            j = 0;
                            do {
                                ++s;
                            } while (s_pref[s + 1] == s_pref[s]);
                        }
                        nxt = fetch_block(ix, s_lo[s] + j);
                    }
                    uint32_t id[4], cnt_b;
                    decode_fetched(cur, stage[warp], id, cnt_b);
                    or_tile(tile, lo_id, SPAN, id, cnt_b);
                }
            }
            if (tid == 0) s_ndense = 0;
            __syncthreads();
        }
        if (a.vec_ok) {
            uint4* d4 = reinterpret_cast<uint4*>(dst);
            for (uint32_t j = tid; j * 4u + 3u < nw; j += NT) d4[j] = tile4[j];
            for (uint32_t i = (nw & ~3u) + tid; i < nw; i += NT) dst[i] = tile[i];
        } else {
            for (uint32_t i = tid; i < nw; i += NT) dst[i] = tile[i];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// list-union, dense group variant: one CTA per SM walks 64- or 32-word
// tiles; for each tile, a 2-D TMA copy stages that tile's slice of every
// dense bitmap in shared memory once (double-buffered where two stages fit:
// the next tile's copy is in flight while this one is merged), then every
// non-probe query of the batch ORs its dense slices from shared memory and
// writes its tile (the merge kernel later adds the lists without dense
// bitmaps that a query merges). Dense bitmaps shared by many queries are
// read from L2 / HBM once per tile instead of once per query and tile.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

constexpr uint32_t kGroupThreads = 1024;

// What one lane ORs per row: one word of a 32-word tile, two of a 64-word one.
template <uint32_t GW> struct GroupWord;
template <> struct GroupWord<32> { typedef uint32_t T; };
template <> struct GroupWord<64> { typedef uint2 T; };
__device__ __forceinline__ uint32_t orw(uint32_t a, uint32_t b) { return a | b; }
__device__ __forceinline__ uint2 orw(uint2 a, uint2 b) { return make_uint2(a.x | b.x, a.y | b.y); }
template <typename T> __device__ __forceinline__ T zero_word();
template <> __device__ __forceinline__ uint32_t zero_word<uint32_t>() { return 0u; }
template <> __device__ __forceinline__ uint2 zero_word<uint2>() { return make_uint2(0u, 0u); }
__device__ __forceinline__ bool all_ones(uint32_t a) { return a == ~0u; }
__device__ __forceinline__ bool all_ones(uint2 a) { return (a.x & a.y) == ~0u; }
// true when the warp's whole tile slice is set: no further row can change it
template <typename T>
__device__ __forceinline__ bool tile_full(T acc) { return __all_sync(kFull, all_ones(acc)); }

// Row `woff` (a word offset, row * GW) of a stage, at this lane's column
// (B = stage + lane * GW / 32 words)
template <typename T>
__device__ __forceinline__ T ld_row(const uint8_t* B, uint32_t woff) {
    return *reinterpret_cast<const T*>(B + (woff << 2));
}
// OR of the 8 rows named by the 16-bit word offsets in v
template <typename T>
__device__ __forceinline__ T or8w(const uint8_t* B, uint4 v) {
    return orw(orw(orw(ld_row<T>(B, v.x & 0xffffu), ld_row<T>(B, v.x >> 16)),
                   orw(ld_row<T>(B, v.y & 0xffffu), ld_row<T>(B, v.y >> 16))),
               orw(orw(ld_row<T>(B, v.z & 0xffffu), ld_row<T>(B, v.z >> 16)),
                   orw(ld_row<T>(B, v.w & 0xffffu), ld_row<T>(B, v.w >> 16))));
}
// OR over a list of nd word offsets (padded to a multiple of 8 with the
// zero row), 16 at a time: per row one extract, one address, one shared load.
// The lists are in ascending bitmap order, which is longest list first, so a
// tile of a dense query saturates early; the warp stops once every bit of
// its slice is set (about 30 % of the row reads on config c1).
template <typename T>
__device__ __forceinline__ T or_list_words(const uint8_t* B, const uint4* ol, uint32_t nd) {
    T acc = zero_word<T>();
    uint32_t k = 0;
    for (; k + 16u <= nd; k += 16u) {
        acc = orw(acc, orw(or8w<T>(B, ol[k >> 3]), or8w<T>(B, ol[(k >> 3) + 1])));
        if (tile_full(acc)) return acc;
    }
    if (k < nd) acc = orw(acc, or8w<T>(B, ol[k >> 3]));
    if (k + 8u < nd) acc = orw(acc, or8w<T>(B, ol[(k >> 3) + 1]));
    return acc;
}
// the same over a list of 16-bit row indices read from global memory (used
// when the batch's lists do not fit in shared memory)
template <uint32_t GW, typename T>
__device__ __forceinline__ T or_list_rows(const uint8_t* B, const uint4* dl, uint32_t nd) {
    T acc = zero_word<T>();
    for (uint32_t k = 0; k < nd; k += 8u) {
        const uint4 v = dl[k >> 3];
        const uint4 wv = make_uint4((v.x & 0xffffu) * GW | ((v.x >> 16) * GW) << 16,
                                    (v.y & 0xffffu) * GW | ((v.y >> 16) * GW) << 16,
                                    (v.z & 0xffffu) * GW | ((v.z >> 16) * GW) << 16,
                                    (v.w & 0xffffu) * GW | ((v.w >> 16) * GW) << 16);
        acc = orw(acc, or8w<T>(B, wv));
        if (tile_full(acc)) break;
    }
    return acc;
}

// Shared memory (dynamic, 1024-byte aligned base): two stages of n_rows x
// GW words (rows = dense bitmaps + the zero row), then per such query
// its list's offset and length, the queue of those queries, and the
// lists themselves as 16-bit row word offsets (row * GW) when they fit (else
// the 16-bit row lists are read from global memory). GW = 64 halves the
// index work per word (each lane ORs two words per row) where two stages of
// 64-word rows fit.
template <uint32_t GW>
__global__ void __launch_bounds__(kGroupThreads, 1)
    dense_group_kernel(const __grid_constant__ CUtensorMap tmap_full, const __grid_constant__ CUtensorMap tmap_last,
                       DenseGroupArgs a) {
    typedef typename GroupWord<GW>::T T;
    constexpr uint32_t kLaneWords = GW / 32u;
    static_assert(kGroupMaxBoxes * kGroupBoxRows * GW < 65536u, "16-bit word offsets");
    extern __shared__ uint8_t g_raw[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t s_next[2];
    __shared__ uint32_t s_ndq;
    __shared__ uint32_t s_warp[32];
    uint8_t* base = g_raw + ((1024u - (smem_addr(g_raw) & 1023u)) & 1023u);
    const uint32_t stage_bytes = (a.n_rows * GW * 4u + 1023u) & ~1023u;
    const bool dbl = a.stages == 2u;  // two stages: the next tile's copy overlaps this tile's merge
    uint32_t* stage0 = reinterpret_cast<uint32_t*>(base);
    uint32_t* s_meta = reinterpret_cast<uint32_t*>(base + a.stages * stage_bytes);  // n_q: list offset / 8 << 16 | nd
    uint16_t* s_qlist = reinterpret_cast<uint16_t*>(s_meta + a.n_q);               // queries with q_dmode != 0
    uint4* s_lists = reinterpret_cast<uint4*>(base + a.stages * stage_bytes + ((6u * a.n_q + 15u) & ~15u));
    const uint32_t tid = threadIdx.x, lane = lane_id(), warp = warp_id();
    constexpr uint32_t kNW = kGroupThreads / 32u;
    uint32_t t = blockIdx.x;
    if (t >= a.n_tiles) return;
    const uint32_t full_boxes = (a.n_rows - 1u) / kGroupBoxRows;  // boxes of 256 rows before the last
    auto issue = [&](uint32_t tile, uint32_t st) {  // thread 0 only
        fence_proxy_async();  // earlier reads of this stage (ordered by the barrier) before the copy
        mbar_expect_tx(&bar[st], a.n_rows * GW * 4u);
        uint32_t* dst = stage0 + st * (stage_bytes / 4u);
        for (uint32_t j = 0; j < full_boxes; ++j)
            tma_load_2d(dst + j * kGroupBoxRows * GW, &tmap_full, int(tile * GW), int(j * kGroupBoxRows), &bar[st]);
        tma_load_2d(dst + full_boxes * kGroupBoxRows * GW, &tmap_last, int(tile * GW), int(full_boxes * kGroupBoxRows),
                    &bar[st]);
    };
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
        s_next[0] = s_next[1] = 0;
        issue(t, 0);  // the first tile's copy overlaps the list staging below
    }
    // stage those queries' lists (the same for every tile): offsets
    // by a block scan over the queries, at most two per thread
    uint32_t len[2], cnt[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const uint32_t q = tid * 2u + r;
        const bool dq = q < a.n_q && a.q_dmode[q];
        len[r] = dq ? ((a.q_ndense[q] + 7u) & ~7u) : 0u;
        cnt[r] = dq ? 1u : 0u;
    }
    uint32_t tot_len, tot_cnt;
    const uint32_t off0 = block_excl_scan<kGroupThreads>(len[0] + len[1], s_warp, &tot_len);
    const uint32_t rk0 = block_excl_scan<kGroupThreads>(cnt[0] + cnt[1], s_warp, &tot_cnt);
    const bool in_smem = tot_len <= a.list_cap;
    {
        uint32_t off = off0, rk = rk0;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const uint32_t q = tid * 2u + r;
            if (q < a.n_q) s_meta[q] = cnt[r] ? ((off >> 3) << 16) | a.q_ndense[q] : 0xffffffffu;
            if (cnt[r]) s_qlist[rk] = uint16_t(q);
            off += len[r];
            rk += cnt[r];
        }
    }
    if (tid == 0) s_ndq = tot_cnt;
    __syncthreads();
    if (in_smem) {
        constexpr uint32_t kShift = GW == 64u ? 6u : 5u;  // row -> word offset, both halves at once
        for (uint32_t i = warp; i < tot_cnt; i += kNW) {  // a warp per query, 16 bytes per lane
            const uint32_t q = s_qlist[i];
            const uint32_t m = s_meta[q];
            const uint4* src = reinterpret_cast<const uint4*>(a.q_dense16 + a.q_dstart[q]);
            uint4* dst = s_lists + (m >> 16);
            for (uint32_t j = lane; j < ((m & 0xffffu) + 7u) / 8u; j += 32u) {
                const uint4 v = src[j];
                dst[j] = make_uint4(v.x << kShift, v.y << kShift, v.z << kShift, v.w << kShift);
            }
        }
    }
    __syncthreads();
    const uint32_t n_dq = s_ndq;
    uint32_t phase = 0;  // bit s: parity of stage s's next completion
    for (uint32_t it = 0; t < a.n_tiles; ++it, t += gridDim.x) {
        const uint32_t st = dbl ? (it & 1u) : 0u;
        const bool more = t + gridDim.x < a.n_tiles;
        const uint32_t par = (phase >> st) & 1u;
        const bool ok = mbar_wait_bounded(&bar[st], par, a.spin_limit);
        if (__syncthreads_or(!ok)) {
            // The copy into this stage is the only one in flight: the next
            // tile's copy is issued only after a wait succeeds. It gets one
            // more bounded interval to land before the CTA (and its shared
            // memory) goes; a copy still pending after that is abandoned
            // with the error bit set.
            if (tid == 0) atomicOr(a.err, kErrTmaTimeout);
            mbar_wait_bounded(&bar[st], par, a.spin_limit);
            return;
        }
        phase ^= 1u << st;
        // the other stage was released by the barrier that ended the previous
        // tile: its refill overlaps this tile's merge
        if (tid == 0 && more && dbl) issue(t + gridDim.x, st ^ 1u);
        const uint32_t* S = stage0 + st * (stage_bytes / 4u);
        const uint8_t* B = reinterpret_cast<const uint8_t*>(S + lane * kLaneWords);
        const uint64_t w = uint64_t(t) * GW + lane * kLaneWords;
        for (;;) {
            uint32_t i = 0;
            if (lane == 0) i = atomicAdd(&s_next[st], 1u);
            i = __shfl_sync(kFull, i, 0);
            if (i >= n_dq) break;
            const uint32_t q = s_qlist[i];
            const uint32_t m = s_meta[q];
            const uint32_t nd = m & 0xffffu;
            const T acc = in_smem ? or_list_words<T>(B, s_lists + (m >> 16), nd)
                                  : or_list_rows<GW, T>(B, reinterpret_cast<const uint4*>(a.q_dense16 + a.q_dstart[q]),
                                                        nd);
            uint32_t* o = a.out + uint64_t(q) * a.out_stride + w;
            if (a.sat && tile_full(acc) && lane == 0)
                atomicOr(a.sat + uint64_t(q) * a.sat_stride + (t >> 5), 1u << (t & 31u));
            if constexpr (GW == 64u) {
                if (w + 1u < a.n_words) *reinterpret_cast<uint2*>(o) = acc;  // 8-byte aligned (checked at launch)
                else if (w < a.n_words) o[0] = acc.x;
            } else {
                if (w < a.n_words) o[0] = acc;
            }
        }
        __syncthreads();  // this stage is read; the next iteration may refill it
        if (tid == 0) {
            s_next[st] = 0;
            // one stage: the next tile's copy starts now that every warp is
            // done with this one (the arrive in issue() publishes the reset)
            if (!dbl && more) issue(t + gridDim.x, 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// list-union, scatter variant (load-balanced over the short lists' blocks)
// ---------------------------------------------------------------------------
template <int NW>
__global__ void __launch_bounds__(NW * 32) scatter_kernel(IndexView ix, ScatterArgs a) {
    __shared__ __align__(16) uint4 stage[NW][32];
    const uint32_t warp = warp_id();
    const uint64_t total = a.q_light_pref[a.n_q];
    const uint64_t bpw = a.blocks_per_warp;
    const uint64_t nwt = uint64_t(gridDim.x) * NW;
    for (uint64_t f0 = (uint64_t(blockIdx.x) * NW + warp) * bpw; f0 < total; f0 += nwt * bpw) {
        const uint64_t f1 = f0 + bpw < total ? f0 + bpw : total;
        // query: last q with q_light_pref[q] <= f0
        uint32_t q0 = 0, q1 = a.n_q;
        while (q1 - q0 > 1) {
            const uint32_t m = (q0 + q1) >> 1;
            if (a.q_light_pref[m] <= f0) q0 = m; else q1 = m;
        }
        uint32_t q = q0;
        uint64_t qb = a.q_off[q], qe = a.q_off[q + 1];
        uint32_t qtot = uint32_t(a.q_light_pref[q + 1] - a.q_light_pref[q]);
        const uint32_t r = uint32_t(f0 - a.q_light_pref[q]);
        // term slot: last i with term_lpref[i] <= r
        uint64_t i0 = qb, i1 = qe;
        while (i1 - i0 > 1) {
            const uint64_t m = (i0 + i1) >> 1;
            if (a.term_lpref[m] <= r) i0 = m; else i1 = m;
        }
        uint64_t i = i0;
        uint32_t j = r - a.term_lpref[i];
        uint32_t* out = a.out + uint64_t(a.out_slot ? a.out_slot[q] : q) * a.out_stride;
        const uint32_t* sat = a.sat ? a.sat + uint64_t(q) * a.sat_stride : nullptr;
        // (i, j) is a scattered block of query q; the walk moves to the next
        // one, crossing into later terms and queries as they run out
        auto advance = [&]() {
            ++j;
            for (;;) {
                const uint32_t nb = (i + 1 < qe ? a.term_lpref[i + 1] : qtot) - a.term_lpref[i];
                if (j < nb) return;
                ++i;
                j = 0;
                if (i >= qe) {
                    do {
                        ++q;
                    } while (a.q_light_pref[q + 1] == a.q_light_pref[q]);
                    qb = a.q_off[q];
                    qe = a.q_off[q + 1];
                    qtot = uint32_t(a.q_light_pref[q + 1] - a.q_light_pref[q]);
                    i = qb;
                    out = a.out + uint64_t(a.out_slot ? a.out_slot[q] : q) * a.out_stride;
                    if (a.sat) sat = a.sat + uint64_t(q) * a.sat_stride;
                }
            }
        };
        // exclusive bound on the ids of block b, the j-th of slot i: the next
        // block's first id, or n_ads after the term's last block (only
        // needed with saturation marks)
        auto block_hi = [&](uint32_t b) -> uint32_t {
            if (!a.sat) return ix.n_ads;
            const uint32_t nb = (i + 1 < qe ? a.term_lpref[i + 1] : qtot) - a.term_lpref[i];
            return j + 1u < nb ? __ldg(ix.blk_first + b + 1u) : ix.n_ads;
        };
        uint32_t b = __ldg(ix.term_blk + a.terms[i]) + j;
        Fetched nxt = fetch_block(ix, b);
        uint32_t nxt_hi = block_hi(b);
        uint32_t* nxt_out = out;
        const uint32_t* nxt_sat = sat;
        for (uint64_t f = f0; f < f1; ++f) {
            const Fetched cur = nxt;
            const uint32_t cur_hi = nxt_hi;
            uint32_t* cur_out = nxt_out;
            const uint32_t* cur_sat = nxt_sat;
            if (f + 1 < f1) {  // next block's loads in flight during this decode
                advance();
                b = __ldg(ix.term_blk + a.terms[i]) + j;
                nxt = fetch_block(ix, b);
                nxt_hi = block_hi(b);
                nxt_out = out;
                nxt_sat = sat;
            }
            // a block whose whole id range lies in tiles the dense lists
            // already filled changes nothing: skip its decode and ORs
            if (cur_sat && range_saturated(cur_sat, a.sat_shift, cur.first, cur_hi)) continue;
            uint32_t id[4], cnt;
            decode_fetched(cur, stage[warp], id, cnt);
            or_global(cur_out, ix.n_ads, id, cnt, cur_sat, a.sat_shift);
        }
    }
}

// ---------------------------------------------------------------------------
// bitmap-probe
// ---------------------------------------------------------------------------
template <int NW>
__global__ void __launch_bounds__(NW * 32) probe_kernel(IndexView ix, ProbeArgs a) {
    __shared__ __align__(128) uint32_t sbm[kProbeSmemWords];
    __shared__ __align__(16) uint4 stage[NW][32];
    __shared__ __align__(8) uint64_t bar;
    const uint32_t tid = threadIdx.x, lane = lane_id(), warp = warp_id();
    // the device counter also counts queries demoted past the slot capacity
    uint32_t n_probe = a.n_probe_host;
    if (a.d_n_probe && *a.d_n_probe < n_probe) n_probe = *a.d_n_probe;
    if (n_probe == 0 || ix.n_blocks == 0) return;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    const uint64_t cb = a.chunk_blocks;
    const uint64_t n_chunks = (ix.n_blocks + cb - 1) / cb;
    for (uint64_t chunk = blockIdx.x; chunk < n_chunks; chunk += gridDim.x) {
        const uint64_t c0 = chunk * cb;
        const uint64_t c1 = c0 + cb < ix.n_blocks ? c0 + cb : ix.n_blocks;
        const uint32_t t0 = __ldg(ix.blk_term + c0), t1 = __ldg(ix.blk_term + c1 - 1);
        const uint32_t w0 = (t0 >> 5) & ~3u;
        uint32_t w1 = ((t1 >> 5) + 4u) & ~3u;
        if (w1 > a.qbm_words) w1 = a.qbm_words;
        const uint32_t span = w1 > w0 ? w1 - w0 : 0u;
        for (uint32_t g0 = 0; g0 < n_probe; g0 += kProbeGroup) {
            const uint32_t G = n_probe - g0 < kProbeGroup ? n_probe - g0 : kProbeGroup;
            const bool staged = a.staged_ok && span > 0 && (span & 3u) == 0 && span * G <= kProbeSmemWords;
            if (staged) {
                __syncthreads();  // everyone is done with the previous slice
                if (tid == 0) {
                    fence_proxy_async();
                    mbar_expect_tx(&bar, span * 4u * G);
                    for (uint32_t g = 0; g < G; ++g)
                        bulk_g2s(sbm + g * span, a.qbm + uint64_t(g0 + g) * a.qbm_stride + w0, span * 4u, &bar);
                }
                const bool ok = mbar_wait_bounded(&bar, phase, a.spin_limit);
                if (__syncthreads_or(!ok)) {
                    // one more bounded interval for the copies to land before
                    // the CTA's shared memory is released; copies still
                    // pending after it are abandoned with the error bit set
                    if (tid == 0) atomicOr(a.err, kErrTmaTimeout);
                    mbar_wait_bounded(&bar, phase, a.spin_limit);
                    return;
                }
                phase ^= 1u;
            }
            for (uint64_t base = c0 + uint64_t(warp) * 128u; base < c1; base += uint64_t(NW) * 128u) {
                const uint64_t idx = base + lane * 4u;
                uint32_t tv[4];
                if (idx + 3 < c1) {
                    const uint4 v = __ldg(reinterpret_cast<const uint4*>(ix.blk_term + idx));
                    tv[0] = v.x; tv[1] = v.y; tv[2] = v.z; tv[3] = v.w;
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) tv[k] = idx + k < c1 ? __ldg(ix.blk_term + idx + k) : kFull;
                }
                uint32_t hit[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    uint32_t m = 0;
                    const uint32_t term = tv[k];
                    if (term != kFull) {
                        const uint32_t wd = term >> 5, bit = term & 31u;
                        if (wd < a.qbm_words) {
                            for (uint32_t g = 0; g < G; ++g) {
                                const uint32_t word = staged ? sbm[g * span + (wd - w0)]
                                                             : __ldg(a.qbm + uint64_t(g0 + g) * a.qbm_stride + wd);
                                m |= ((word >> bit) & 1u) << g;
                            }
                        }
                    }
                    hit[k] = m;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    uint32_t lanes = __ballot_sync(kFull, hit[k] != 0u);
                    while (lanes) {
                        const uint32_t src = __ffs(lanes) - 1u;
                        lanes &= lanes - 1u;
                        uint32_t qm = __shfl_sync(kFull, hit[k], src);
                        const uint32_t b = uint32_t(base + src * 4u + k);
                        uint32_t id[4], cnt;
                        decode_block(ix, b, stage[warp], id, cnt);
                        while (qm) {
                            const uint32_t g = __ffs(qm) - 1u;
                            qm &= qm - 1u;
                            const uint32_t slot = g0 + g;
                            const uint32_t o = a.out_slot ? a.out_slot[slot] : slot;
                            or_global(a.out + uint64_t(o) * a.out_stride, ix.n_ads, id, cnt);
                        }
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// compaction: one pass (chunk popcount, decoupled look-back, id writes)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t masked_word(const uint32_t* bm, uint64_t w, uint64_t n_bits) {
    uint32_t v = bm[w];
    const uint64_t lo = w * 32u;
    if (lo + 32u > n_bits) v &= (n_bits > lo) ? ((1u << uint32_t(n_bits - lo)) - 1u) : 0u;
    return v;
}

__device__ __forceinline__ uint64_t ld_status(const uint64_t* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
// A status word carries its own value, and no other write of a work item is
// read by another CTA while the kernel runs, so publishing needs no fence:
// one atomic exchange at L2, where the look-back's volatile loads read it.
__device__ __forceinline__ void st_status(uint64_t* p, uint64_t v) {
    atomicExch(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

// Decoupled look-back, run by one whole warp for work item `item` whose own
// id count is `agg`: publishes the count, then reads the status words of the
// earlier items 32 at a time (lane k reads item - 1 - k of the window),
// waits until none of them is empty, and adds up the counts back to the
// nearest item that has published its inclusive prefix; publishes its own
// inclusive prefix and returns the exclusive one in *excl. Items are claimed
// in ascending order by running CTAs, each of which publishes its count
// before it looks back, so every wait ends; a wait that still sees an empty
// word after `limit` polls gives up and returns false.
__device__ bool lookback_prefix(uint64_t* status, uint64_t item, uint32_t agg, uint32_t limit, uint64_t* excl) {
    const uint32_t lane = lane_id();
    if (item == 0) {
        if (lane == 0) st_status(status, kFlagIncl | agg);
        *excl = 0;
        return true;
    }
    if (lane == 0) st_status(status + item, kFlagAgg | agg);
    uint64_t prefix = 0;
    uint64_t end = item;  // the window is items [end - 32, end)
    uint32_t spins = 0;
    for (;;) {
        const bool in_range = end > uint64_t(lane);
        const uint64_t sw = in_range ? ld_status(status + (end - 1u - lane)) : kFlagIncl;  // before item 0: 0
        if (__any_sync(kFull, (sw >> 62) == 0u)) {
            if (++spins > limit) {
                *excl = prefix;
                return false;
            }
            __nanosleep(64);
            continue;
        }
        const uint32_t incl = __ballot_sync(kFull, (sw >> 62) == 2u);
        const uint32_t upto = incl ? uint32_t(__ffs(incl)) - 1u : 31u;  // nearest inclusive word in the window
        uint64_t v = lane <= upto ? (sw & kValMask) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        prefix += v;
        if (incl) break;
        end -= 32u;
    }
    if (lane == 0) st_status(status + item, kFlagIncl | (prefix + agg));
    *excl = prefix;
    return true;
}

// One CTA per (bitmap, 1024-word chunk) at a time, items taken in ascending
// order from a ticket counter. Each of the 4 warps owns 8 consecutive units
// of 32 words, held in registers (lane l: word l of each unit); the chunk's
// id count is published and its output offset found by a decoupled
// look-back before the CTA starts it, and then every warp expands its units
// on its own into ascending ids (three expansions by the unit's id count,
// below). The bitmap is read once: there is no separate counting pass.
constexpr uint32_t kUnits = kCompactChunkWords / 32;
constexpr uint32_t kWarpUnits = kUnits / kCompactWarps;
static_assert(kWarpUnits == 8, "each warp covers 8 units of its CTA's chunk");

// bulk copy shared -> global (TMA engine), completion tracked per thread
__device__ __forceinline__ void bulk_s2g(void* gdst, const void* ssrc, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_addr(ssrc)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

constexpr uint32_t kIdBuf = 1024 + 8;  // one unit's ids plus the 16-byte alignment head

// Ids of one unit into dst[0 .. tot): lane l holds word l of the unit in v
// and the ids of the lower lanes' words in ex; id0 = first id of the unit +
// lane. Three expansions, by the unit's id count t:
//  * t >= kPairMin: two bits per lane -- lanes 0-15 take bits 2j, 2j+1 of
//    the even word, lanes 16-31 those of the odd word, so one pair of
//    shuffles serves two words; a lane stores at most two ids per step.
//  * t < kPairMin: each lane writes the ids of its own word, lowest bit
//    first, for as many steps as the fullest word of the unit has bits;
//    no shuffles, and a sparse unit costs steps in proportion to its bits.
//  * t == 1024 (every bit set) is handled by the caller without bit work.
// Measured on bitmaps with the per-query densities of config c1: 6 % less
// time than one lane per bit for every dense unit and a shuffle loop over
// the non-zero words for the rest, and 2x at 25 % density.
constexpr uint32_t kPairMin = 384;

template <typename Store>
__device__ __forceinline__ void expand_pairs(uint32_t v, uint32_t ex, uint32_t id0, Store store) {
    const uint32_t lane = lane_id();
    const uint32_t half = lane >> 4, j = lane & 15u;
    const uint32_t below = (1u << (2u * j)) - 1u;               // bits under this lane's pair
    const uint32_t base = id0 - lane + half * 32u + 2u * j;     // id of bit 2j of word `half`
#pragma unroll 4
    for (uint32_t i = 0; i < 16u; ++i) {
        const uint32_t w = 2u * i + half;
        const uint32_t word = __shfl_sync(kFull, v, w);
        const uint32_t pos = __shfl_sync(kFull, ex, w);
        const uint32_t b2 = (word >> (2u * j)) & 3u;
        const uint32_t p = pos + __popc(word & below);
        const uint32_t id = base + i * 64u;
        if (b2 & 1u) store(p, id);
        if (b2 & 2u) store(p + (b2 & 1u), id + 1u);
    }
}

template <typename Store>
__device__ __forceinline__ void expand_lane_word(uint32_t v, uint32_t ex, uint32_t id0, Store store) {
    const uint32_t lane = lane_id();
    const uint32_t wb = id0 - lane + 32u * lane;  // id of bit 0 of this lane's word
    const uint32_t steps = __reduce_max_sync(kFull, uint32_t(__popc(v)));
    uint32_t w = v, p = ex;
    for (uint32_t i = 0; i < steps; ++i) {
        if (w) {
            store(p, wb + uint32_t(__ffs(w)) - 1u);
            ++p;
            w &= w - 1u;
        }
    }
}

// async 4-byte copy global -> shared (LDGSTS: no register round trip)
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// One warp claims the next work item and makes it ready for the CTA: the
// chunk's words into buf (lane l: word 32 m + l), each warp slice's id count
// into s_wtot, the decoupled look-back's exclusive prefix into *s_prefix.
// The claim is followed at once by the loads and the count's publication, so
// later items' look-backs never wait long on it.
__device__ void prepare_chunk(const CompactArgs& a, uint64_t items, uint64_t n_words, uint32_t* buf,
                              unsigned long long* s_item, unsigned long long* s_prefix, uint32_t* s_wtot) {
    const uint32_t lane = lane_id();
    unsigned long long n = 0;
    if (lane == 0) n = atomicAdd(a.ticket, 1ull);
    n = __shfl_sync(kFull, n, 0);
    if (lane == 0) *s_item = n;
    if (n >= items) return;
    const uint32_t q = uint32_t(n / a.n_chunks);
    const uint32_t c = uint32_t(n - uint64_t(q) * a.n_chunks);
    const uint32_t* bm = a.bm + uint64_t(q) * a.stride;
    const uint64_t wbase = uint64_t(c) * kCompactChunkWords;
#pragma unroll 8
    for (uint32_t m = 0; m < kUnits; ++m) {
        const uint64_t wi = wbase + m * 32u + lane;
        if (wi + 1u < n_words) cp_async4(buf + m * 32u + lane, bm + wi);
        else buf[m * 32u + lane] = wi < n_words ? masked_word(bm, wi, a.n_bits) : 0u;
    }
    cp_async_wait_all();
    __syncwarp();
    uint32_t t = 0;
#pragma unroll
    for (uint32_t w = 0; w < kCompactWarps; ++w) {
        uint32_t cw = 0;
#pragma unroll
        for (uint32_t k = 0; k < kWarpUnits; ++k) cw += __popc(buf[(w * kWarpUnits + k) * 32u + lane]);
        cw = __reduce_add_sync(kFull, cw);
        if (lane == 0) s_wtot[w] = cw;
        t += cw;
    }
    uint64_t excl = 0;
    const bool ok = lookback_prefix(a.status, n, t, a.spin_limit, &excl);
    if (lane == 0) {
        if (!ok) atomicOr(a.err, kErrScanTimeout);
        *s_prefix = excl;
        if (a.id_offsets) {
            if (c == 0) a.id_offsets[q] = excl;
            if (n + 1 == items) a.id_offsets[a.n_q] = excl + t;
        }
        if (a.id_counts && t) atomicAdd(reinterpret_cast<unsigned long long*>(a.id_counts + q), t);
    }
}

// The CTA works on one item while the first of its warps to finish prepares
// the next one in its own id buffer (claim, loads, count, look-back), so the
// claim's round trip, the loads and the look-back overlap the other warps'
// expansion instead of stalling the whole CTA.
__global__ void __launch_bounds__(kCompactWarps * 32, 48 / kCompactWarps) compact_kernel(CompactArgs a) {
    __shared__ __align__(16) uint32_t s_buf[kCompactWarps][kIdBuf];
    __shared__ uint32_t s_wtot[kCompactWarps];
    __shared__ unsigned long long s_item, s_prefix;
    __shared__ uint32_t s_src, s_first;
    static_assert(kCompactChunkWords <= kIdBuf, "a chunk fits one id buffer");
    const uint32_t lane = lane_id(), warp = warp_id();
    const bool ids16 = (reinterpret_cast<uintptr_t>(a.ids) & 15u) == 0;
    uint32_t* buf = s_buf[warp];
    const uint64_t n_words = (a.n_bits + 31) / 32;
    const uint64_t items = uint64_t(a.n_q) * a.n_chunks;
    if (warp == 0) prepare_chunk(a, items, n_words, buf, &s_item, &s_prefix, s_wtot);
    if (threadIdx.x == 0) {
        s_src = 0;
        s_first = 0;
    }
    __syncthreads();
    for (;;) {
        const uint64_t item = s_item;
        if (item >= items) break;
        const uint32_t q = uint32_t(item / a.n_chunks);
        const uint32_t c = uint32_t(item - uint64_t(q) * a.n_chunks);
        const uint64_t wbase = uint64_t(c) * kCompactChunkWords + uint64_t(warp) * (kWarpUnits * 32u);
        const uint32_t* src = s_buf[s_src] + warp * (kWarpUnits * 32u);
        uint32_t v[kWarpUnits], tot[kWarpUnits];
#pragma unroll
        for (uint32_t k = 0; k < kWarpUnits; ++k) {
            v[k] = src[k * 32u + lane];
            tot[k] = __reduce_add_sync(kFull, uint32_t(__popc(v[k])));
        }
        uint64_t o0 = s_prefix + __reduce_add_sync(kFull, lane < warp ? s_wtot[lane] : 0u);
        // every warp holds its words and offset: the chunk's buffer and the
        // next item's slots may be reused
        __syncthreads();
#pragma unroll 1
        for (uint32_t k = 0; k < kWarpUnits; ++k) {
            // a rolled loop keeps one copy of the expansion code (the
            // instruction cache holds it): the current unit is always in
            // v[0], the later ones move down one register per step
            const uint32_t vk = v[0], t = tot[0];
#pragma unroll
            for (uint32_t j = 0; j + 1 < kWarpUnits; ++j) {
                v[j] = v[j + 1];
                tot[j] = tot[j + 1];
            }
            if (t == 0) continue;
            const uint32_t cnt = __popc(vk);
            uint32_t x = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, x, o);
                if (lane >= uint32_t(o)) x += y;
            }
            const uint32_t ex = x - cnt;
            const uint32_t id0 = uint32_t((wbase + k * 32u) * 32u) + lane;
            uint32_t* dst = a.ids + o0;
            if (ids16 && o0 + t <= a.capacity) {
                // the unit's ids go to the warp's shared buffer at their
                // 16-byte-aligned output position; the aligned middle leaves
                // by one bulk copy, the ragged ends by plain stores
                const uint32_t head = uint32_t(o0 & 3u);
                uint32_t* sb = buf + head;
                if (lane == 0) bulk_wait_read_all();  // the previous unit's copy has read the buffer
                __syncwarp();
                auto st = [sb](uint32_t i, uint32_t id) { sb[i] = id; };
                if (t == 1024u) {
                    // every bit set: buf[x] = first id of the unit + x - head
                    const uint32_t b0 = id0 - lane - head;
                    uint4* b4 = reinterpret_cast<uint4*>(buf);
#pragma unroll
                    for (uint32_t m = lane; m < kIdBuf / 4u; m += 32u) {
                        const uint32_t x = b0 + 4u * m;
                        b4[m] = make_uint4(x, x + 1u, x + 2u, x + 3u);
                    }
                } else if (t >= kPairMin) {
                    expand_pairs(vk, ex, id0, st);
                } else {
                    expand_lane_word(vk, ex, id0, st);
                }
                fence_proxy_async();  // these shared writes before the async-proxy read
                __syncwarp();
                const uint32_t end = head + t;
                const uint32_t mid_hi = end & ~3u;
                uint32_t* gbase = dst - head;  // 16-byte aligned
                if (lane == 0 && mid_hi > 4u) {
                    bulk_s2g(gbase + 4, buf + 4, (mid_hi - 4u) * 4u);
                    bulk_commit();
                }
                if (lane >= head && lane < 4u && lane < end) gbase[lane] = buf[lane];
                if (mid_hi + lane < end && mid_hi + lane >= 4u) gbase[mid_hi + lane] = buf[mid_hi + lane];
            } else if (o0 + t <= a.capacity) {  // whole unit fits: no per-id check
                expand_lane_word(vk, ex, id0, [dst](uint32_t i, uint32_t id) { dst[i] = id; });
            } else {
                const uint64_t cap = a.capacity;
                const uint64_t ob = o0;
                uint32_t* ids = a.ids;
                expand_lane_word(vk, ex, id0, [=](uint32_t i, uint32_t id) {
                    if (ob + i < cap) ids[ob + i] = id;
                });
            }
            o0 += t;
        }
        // the first warp done prepares the next item in its own buffer
        uint32_t first = 0;
        if (lane == 0) first = atomicAdd(&s_first, 1u);
        first = __shfl_sync(kFull, first, 0);
        if (first == 0) {
            if (lane == 0) bulk_wait_read_all();  // its last copy has read the buffer
            __syncwarp();
            prepare_chunk(a, items, n_words, buf, &s_item, &s_prefix, s_wtot);
            if (lane == 0) s_src = warp;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_first = 0;
    }
    if (lane == 0) bulk_wait_all();
}

// ---------------------------------------------------------------------------
// self-test of the bounded waits
// ---------------------------------------------------------------------------
// CTA 0 arms an mbarrier for 16 bytes that no copy delivers and waits on it
// with mbar_wait_bounded; CTA 1 looks back from item 1 at status[0], which
// nothing publishes, with lookback_prefix. No asynchronous copy is ever
// issued, so nothing is in flight when the CTAs leave.
__global__ void __launch_bounds__(32) wait_selftest_kernel(uint64_t* status2, uint32_t* err, uint32_t limit) {
    __shared__ __align__(8) uint64_t bar;
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            fence_mbar_init();
            mbar_expect_tx(&bar, 16u);
        }
        __syncwarp();
        const bool ok = mbar_wait_bounded(&bar, 0u, limit);
        if (__any_sync(kFull, !ok) && threadIdx.x == 0) atomicOr(err, kErrTmaTimeout);
    } else {
        uint64_t excl = 0;
        const bool ok = lookback_prefix(status2, 1u, 7u, limit, &excl);
        if (!ok && threadIdx.x == 0) atomicOr(err, kErrScanTimeout);
    }
}

inline int grid_for(uint64_t items, int sm_count, uint32_t per_sm) {
    uint64_t g = uint64_t(sm_count) * (per_sm ? per_sm : 1u);
    if (items < g) g = items;
    return int(g ? g : 1);
}

}  // namespace

IndexView view_of(const abf_index* ix) {
    IndexView v;
    v.payload = reinterpret_cast<const uint4*>(ix->dev.payload);
    v.blk_first = ix->dev.blk_first;
    v.blk_last = ix->dev.blk_last;
    v.blk_desc = reinterpret_cast<const uint2*>(ix->dev.blk_desc);
    v.blk_term = ix->dev.blk_term;
    v.term_blk = ix->dev.term_blk;
    v.term_len = ix->dev.term_len;
    v.term_dense = ix->dev.term_dense;
    v.dense = ix->dev.dense;
    v.term_dir = ix->dev.term_dir;
    v.dir = ix->dev.dir;
    v.term_cbytes = ix->dev.term_cbytes;
    v.dense_stride = ix->derived.dense_stride;
    v.dir_n = ix->derived.dir_n;
    v.n_dense = ix->derived.n_dense;
    v.n_terms = ix->n_terms;
    v.n_ads = ix->n_ads;
    v.n_blocks = ix->n_blocks;
    return v;
}

uint32_t compact_chunks(uint64_t n_bits) {
    const uint64_t n_words = (n_bits + 31) / 32;
    return uint32_t((n_words + kCompactChunkWords - 1) / kCompactChunkWords);
}

cudaError_t launch_plan(const IndexView& v, const PlanArgs& a, cudaStream_t s) {
    if (a.n_q == 0) return cudaSuccess;
    const uint32_t g = a.n_q < 65535u * 16u ? a.n_q : 65535u * 16u;
    plan_kernel<<<g, 256, 0, s>>>(v, a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_queue_scan(const QueueArgs& a, cudaStream_t s) {
    queue_scan_kernel<<<1, 1024, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

template <int W, int NW>
static cudaError_t tile_launch(const IndexView& v, const TileArgs& a, int grid, cudaStream_t s) {
    constexpr int smem = W * 4;
    if (smem > 48 * 1024) {
        // opt in to more than 48 KB of dynamic shared memory, once per device
        // (so that later launches, also under stream capture, make no
        // host-side attribute call)
        static std::atomic<uint64_t> done{0};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const uint64_t bit = 1ull << (dev & 63);
        if (!(done.load() & bit)) {
            e = cudaFuncSetAttribute(tile_union_kernel<W, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
            done.fetch_or(bit);
        }
    }
    tile_union_kernel<W, NW><<<grid, NW * 32, smem, s>>>(v, a);
    return cudaGetLastError();
}

template <int W>
static cudaError_t tile_dispatch_w(const IndexView& v, const TileArgs& a, uint32_t nw, int grid, cudaStream_t s) {
    switch (nw) {
        case 1: return tile_launch<W, 1>(v, a, grid, s);
        case 2: return tile_launch<W, 2>(v, a, grid, s);
        case 4: return tile_launch<W, 4>(v, a, grid, s);
        default: return tile_launch<W, 8>(v, a, grid, s);
    }
}

cudaError_t launch_tile_union(const IndexView& v, const TileArgs& a, const abf_tuning& t, int sm_count,
                              cudaStream_t s) {
    const uint64_t items = uint64_t(a.n_q) * a.n_tiles;
    if (items == 0) return cudaSuccess;
    const uint32_t nw = t.warps_per_tile ? t.warps_per_tile : 8u;
    // ctas_per_sm counts 8-warp CTAs; narrower CTAs are packed proportionally
    const uint32_t per_sm = (t.ctas_per_sm ? t.ctas_per_sm : 2u) * (nw >= 8u ? 1u : 8u / nw);
    const int grid = grid_for(items, sm_count, per_sm);
    cudaError_t e;
    switch (t.tile_words) {
        case 256: e = tile_dispatch_w<256>(v, a, nw, grid, s); break;
        case 512: e = tile_dispatch_w<512>(v, a, nw, grid, s); break;
        case 2048: e = tile_dispatch_w<2048>(v, a, nw, grid, s); break;
        case 4096: e = tile_dispatch_w<4096>(v, a, nw, grid, s); break;
        case 8192: e = tile_dispatch_w<8192>(v, a, nw, grid, s); break;
        case 16384: e = tile_dispatch_w<16384>(v, a, nw, grid, s); break;
        default: e = tile_dispatch_w<1024>(v, a, nw, grid, s); break;
    }
    count_launch();
    return e;
}

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encoder() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return EncodeTiledFn(nullptr);
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}
}  // namespace

cudaError_t encode_dense_tmap(const IndexView& v, uint32_t gw, void* out) {
    static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
    EncodeTiledFn fn = encoder();
    if (!fn || !v.dense || v.n_dense == 0 || (gw != 32u && gw != 64u)) return cudaErrorNotSupported;
    // dims: words of a bitmap (innermost), bitmaps; rows past n_dense read as
    // zeros. Two descriptors: boxes of 256 bitmaps, and one box for the rest
    // plus the zero row, so a stage holds exactly n_dense + 1 rows.
    const uint32_t rows = v.n_dense + 1u;
    const uint32_t last = rows - (rows - 1u) / kGroupBoxRows * kGroupBoxRows;
    const cuuint64_t dims[2] = {cuuint64_t(v.dense_stride), cuuint64_t(v.n_dense)};
    const cuuint64_t strides[1] = {cuuint64_t(v.dense_stride) * 4u};
    const cuuint32_t es[2] = {1, 1};
    for (int k = 0; k < 2; ++k) {
        const cuuint32_t box[2] = {gw, k == 0 ? kGroupBoxRows : last};
        const CUresult r = fn(reinterpret_cast<CUtensorMap*>(out) + k, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2,
                              const_cast<uint32_t*>(v.dense), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

uint32_t dense_group_list_cap(uint32_t n_rows, uint32_t n_q, uint32_t gw, uint32_t stages) {
    const uint64_t stage = (uint64_t(n_rows) * gw * 4u + 1023u) & ~1023ull;
    const uint64_t used = 1024u + stages * stage + ((6ull * n_q + 15u) & ~15ull);
    return used >= kGroupSmemBytes ? 0u : uint32_t((kGroupSmemBytes - used) / 2u) & ~7u;
}

namespace {
template <uint32_t GW>
cudaError_t launch_group_w(const CUtensorMap (&m)[2], const DenseGroupArgs& a, int sm_count, cudaStream_t s) {
    static std::atomic<uint64_t> done{0};  // devices whose attribute is set
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!(done.load() >> dev & 1ull)) {
        e = cudaFuncSetAttribute(dense_group_kernel<GW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kGroupSmemBytes));
        if (e != cudaSuccess) return e;
        done.fetch_or(1ull << dev);
    }
    const uint32_t grid = a.n_tiles < uint32_t(sm_count) ? a.n_tiles : uint32_t(sm_count);
    dense_group_kernel<GW><<<grid, kGroupThreads, kGroupSmemBytes, s>>>(m[0], m[1], a);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_dense_group(const void* tmaps, uint32_t gw, const DenseGroupArgs& a, int sm_count,
                               cudaStream_t s) {
    if (a.n_q == 0 || a.n_tiles == 0) return cudaSuccess;
    if (a.n_rows < 2 || a.n_rows > kGroupMaxBoxes * kGroupBoxRows || a.n_q > kGroupMaxQueries)
        return cudaErrorInvalidValue;
    const uint64_t stage = (uint64_t(a.n_rows) * gw * 4u + 1023u) & ~1023ull;
    if ((a.stages != 1u && a.stages != 2u) ||
        1024u + a.stages * stage + ((6ull * a.n_q + 15u) & ~15ull) > kGroupSmemBytes)
        return cudaErrorInvalidValue;
    CUtensorMap m[2];
    std::memcpy(m, tmaps, sizeof(m));
    cudaError_t e;
    if (gw == 64u) e = launch_group_w<64>(m, a, sm_count, s);
    else if (gw == 32u) e = launch_group_w<32>(m, a, sm_count, s);
    else return cudaErrorInvalidValue;
    count_launch();
    return e;
}

cudaError_t launch_scatter(const IndexView& v, const ScatterArgs& a, const abf_tuning& t, int sm_count,
                           cudaStream_t s) {
    if (a.n_q == 0) return cudaSuccess;
    const int grid = grid_for(~0ull, sm_count, t.ctas_per_sm ? t.ctas_per_sm * 2u : 8u);
    scatter_kernel<8><<<grid, 256, 0, s>>>(v, a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_probe(const IndexView& v, const ProbeArgs& a, const abf_tuning& t, int sm_count, cudaStream_t s) {
    if (v.n_blocks == 0) return cudaSuccess;
    const uint64_t n_chunks = (v.n_blocks + a.chunk_blocks - 1) / a.chunk_blocks;
    const int grid = grid_for(n_chunks, sm_count, t.ctas_per_sm ? t.ctas_per_sm : 4u);
    probe_kernel<8><<<grid, 256, 0, s>>>(v, a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_compact(const CompactArgs& a, int sm_count, uint32_t ctas_per_sm, cudaStream_t s) {
    const uint64_t items = uint64_t(a.n_q) * a.n_chunks;
    if (items == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(a.status, 0, items * sizeof(uint64_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.ticket, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess && a.id_counts) e = cudaMemsetAsync(a.id_counts, 0, uint64_t(a.n_q) * sizeof(uint64_t), s);
    if (e != cudaSuccess) return e;
    // ctas_per_sm counts CTAs of 8 warps: the same resident warps whatever the CTA size
    const uint32_t per_sm = (ctas_per_sm ? ctas_per_sm : 6u) * 8u / kCompactWarps;
    compact_kernel<<<grid_for(items, sm_count, per_sm), kCompactWarps * 32, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_wait_selftest(uint64_t* status2, uint32_t* err, uint32_t spin_limit, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(status2, 0, 2 * sizeof(uint64_t), s);
    if (e != cudaSuccess) return e;
    wait_selftest_kernel<<<2, 32, 0, s>>>(status2, err, spin_limit);
    count_launch();
    return cudaGetLastError();
}

}  // namespace abf
