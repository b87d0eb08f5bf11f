// Device side of the learned path planner, shared by the planner kernels
// (abf_planner.cu) and the plan kernel (abf_kernels.cu), which runs the same
// feature + MLP code inline for ABF_PATH_AUTO queries when parameters are
// installed, so a batch pays no separate planner launch.
//
// The MLP is 16 -> 64 -> 64 -> 3 with ReLU; the three outputs predict
// log(microseconds) of the PROBE, UNION and HYBRID paths of one query.
// Parameter layout (ABF_PLANNER_PARAMS floats, include/adabool.h):
//   mu[16] sd[16] | W1[64][16] b1[64] | W2[64][64] b2[64] | W3[3][64] b3[3]
#pragma once

#include "abf_kernels.cuh"

namespace abf {
namespace plan_dev {
namespace {

constexpr int F = ABF_PLANNER_FEATURES;
constexpr int H = ABF_PLANNER_HIDDEN;
constexpr int O = ABF_PLANNER_OUTPUTS;
constexpr int kMu = 0, kSd = 16, kW1 = 32, kB1 = kW1 + H * F, kW2 = kB1 + H, kB2 = kW2 + H * H, kW3 = kB2 + H,
              kB3 = kW3 + O * H, kNParams = kB3 + O;
static_assert(kNParams == ABF_PLANNER_PARAMS, "parameter layout");
constexpr int kFeatThreads = 256;
constexpr int kFeatUnroll = 4;  // terms per thread per pass, their loads in flight together

__device__ __forceinline__ uint32_t lane() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ uint32_t warp_max(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

struct FeatCtx {
    uint32_t hybrid_min;
    uint64_t n_postings;
    uint32_t n_q;
};

// The 16 features of query q, computed by the whole CTA (kFeatThreads
// threads) into f[] in shared memory. Term ids >= n_terms are skipped;
// repeated terms count once per occurrence. Each thread takes kFeatUnroll
// terms per pass and issues all their table loads before using any, so a
// query of thousands of terms costs a few memory latencies, not one per term.
__device__ void query_features(const IndexView& ix, const uint32_t* terms, const uint64_t* q_off, uint32_t q,
                               const FeatCtx& c, float* f) {
    __shared__ double s_d[6][kFeatThreads / 32];
    __shared__ uint32_t s_u[4][kFeatThreads / 32];
    const uint64_t qb = q_off[q], qe = q_off[q + 1];
    uint32_t n = 0, mx = 0, nd = 0, nl = 0;
    double S = 0, Q = 0, Cb = 0, Lg = 0, Sd = 0, Bnd = 0;
    const double inv_ads = 1.0 / double(ix.n_ads);
    for (uint64_t i0 = qb + threadIdx.x; i0 < qe; i0 += uint64_t(kFeatThreads) * kFeatUnroll) {
        uint32_t t[kFeatUnroll], len[kFeatUnroll], dn[kFeatUnroll], cb[kFeatUnroll], b0[kFeatUnroll],
            b1[kFeatUnroll];
#pragma unroll
        for (int u = 0; u < kFeatUnroll; ++u) {
            const uint64_t i = i0 + uint64_t(u) * kFeatThreads;
            t[u] = i < qe ? terms[i] : kNone;
        }
#pragma unroll
        for (int u = 0; u < kFeatUnroll; ++u) {
            const bool ok = t[u] < ix.n_terms;
            len[u] = ok ? __ldg(ix.term_len + t[u]) : 0u;
            dn[u] = ok ? __ldg(ix.term_dense + t[u]) : kNone;
            cb[u] = ok ? __ldg(ix.term_cbytes + t[u]) : 0u;
            b0[u] = ok ? __ldg(ix.term_blk + t[u]) : 0u;
            b1[u] = ok ? __ldg(ix.term_blk + t[u] + 1) : 0u;
        }
#pragma unroll
        for (int u = 0; u < kFeatUnroll; ++u) {
            if (t[u] >= ix.n_terms) continue;
            ++n;
            mx = max(mx, len[u]);
            S += len[u];
            Q += double(len[u]) * len[u];
            Cb += cb[u];
            Lg += log1p(-fmin(double(len[u]) * inv_ads, 0.999999));
            if (dn[u] != kNone) {
                ++nd;
                Sd += len[u];
            } else {
                Bnd += b1[u] - b0[u];
                if (len[u] < c.hybrid_min) ++nl;
            }
        }
    }
    const uint32_t w = threadIdx.x >> 5;
    n = warp_sum(n);
    nd = warp_sum(nd);
    nl = warp_sum(nl);
    mx = warp_max(mx);
    S = warp_sum(S);
    Q = warp_sum(Q);
    Cb = warp_sum(Cb);
    Lg = warp_sum(Lg);
    Sd = warp_sum(Sd);
    Bnd = warp_sum(Bnd);
    if (lane() == 0) {
        s_u[0][w] = n; s_u[1][w] = nd; s_u[2][w] = nl; s_u[3][w] = mx;
        s_d[0][w] = S; s_d[1][w] = Q; s_d[2][w] = Cb; s_d[3][w] = Lg; s_d[4][w] = Sd; s_d[5][w] = Bnd;
    }
    __syncthreads();
    // each of the first 16 threads sums the warps' partials and computes one
    // feature (the transcendentals run side by side, not one after another)
    if (threadIdx.x < F) {
        n = nd = nl = mx = 0;
        S = Q = Cb = Lg = Sd = Bnd = 0;
        for (int k = 0; k < kFeatThreads / 32; ++k) {
            n += s_u[0][k]; nd += s_u[1][k]; nl += s_u[2][k]; mx = max(mx, s_u[3][k]);
            S += s_d[0][k]; Q += s_d[1][k]; Cb += s_d[2][k]; Lg += s_d[3][k]; Sd += s_d[4][k]; Bnd += s_d[5][k];
        }
        const double nn = n > 0 ? double(n) : 1.0;
        double r;
        switch (threadIdx.x) {
            case 0: r = log1p(double(n)); break;
            case 1: r = log1p(S); break;
            case 2: r = log1p(double(mx)); break;
            case 3: r = log1p(S / nn); break;
            case 4: {
                const double mean = S / nn;
                r = log1p(sqrt(fmax(Q / nn - mean * mean, 0.0)));
                break;
            }
            case 5: r = log1p(Cb); break;
            case 6: r = 1.0 - exp(Lg); break;
            case 7: r = log1p(double(nd)); break;
            case 8: r = Sd / fmax(S, 1.0); break;
            case 9: r = log1p(Bnd); break;
            case 10: r = S / double(c.n_postings ? c.n_postings : 1); break;
            case 11: r = log1p(double(nl)); break;
            case 12: r = double(q) / double(c.n_q ? c.n_q : 1); break;
            case 13: r = log1p(double(c.n_q)); break;
            case 14: r = double(mx) * inv_ads; break;
            default: r = 1.0; break;
        }
        f[threadIdx.x] = float(r);
    }
    __syncthreads();
}

// MLP forward on standardised x (shared, F floats) by threads 0..63:
// h1, h2 (shared, H each, post-ReLU) and y (shared, O).
__device__ __forceinline__ void mlp_forward_cta(const float* __restrict__ p, const float* xs, float* h1, float* h2,
                                                float* y) {
    const int j = threadIdx.x;
    if (j < H) {
        float a = __ldg(p + kB1 + j);
#pragma unroll
        for (int k = 0; k < F; ++k) a = fmaf(__ldg(p + kW1 + j * F + k), xs[k], a);
        h1[j] = fmaxf(a, 0.0f);
    }
    __syncthreads();
    if (j < H) {
        float a = __ldg(p + kB2 + j);
#pragma unroll 8
        for (int k = 0; k < H; ++k) a = fmaf(__ldg(p + kW2 + j * H + k), h1[k], a);
        h2[j] = fmaxf(a, 0.0f);
    }
    __syncthreads();
    if (j < O) {
        float a = __ldg(p + kB3 + j);
#pragma unroll 8
        for (int k = 0; k < H; ++k) a = fmaf(__ldg(p + kW3 + j * H + k), h2[k], a);
        y[j] = a;
    }
    __syncthreads();
}

// The state the planner keeps in shared memory for one query.
struct PlannerSmem {
    float f[F], xs[F], h1[H], h2[H], y[O];
};

// features -> standardise -> MLP -> cheapest path (an abf_path) of query q,
// by the whole CTA (kFeatThreads threads); sm.f holds the features and sm.y
// the predictions afterwards.
__device__ __forceinline__ uint32_t planner_path(const IndexView& ix, const float* __restrict__ p,
                                                 const uint32_t* terms, const uint64_t* q_off, uint32_t q,
                                                 const FeatCtx& c, PlannerSmem& sm) {
    query_features(ix, terms, q_off, q, c, sm.f);
    if (threadIdx.x < F) {
        const float sd = __ldg(p + kSd + threadIdx.x);
        sm.xs[threadIdx.x] = (sm.f[threadIdx.x] - __ldg(p + kMu + threadIdx.x)) / (sd > 0.0f ? sd : 1.0f);
    }
    __syncthreads();
    mlp_forward_cta(p, sm.xs, sm.h1, sm.h2, sm.y);
    int best = 0;
    for (int o = 1; o < O; ++o)
        if (sm.y[o] < sm.y[best]) best = o;
    return best == 0 ? ABF_PATH_PROBE : best == 1 ? ABF_PATH_UNION : ABF_PATH_HYBRID;
}

}  // namespace
}  // namespace plan_dev
}  // namespace abf
