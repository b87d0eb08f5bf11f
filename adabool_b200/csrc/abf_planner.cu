// Learned path planner: per-query features, the fused feature + MLP
// inference kernel used inside abf_batch_run, and the MLP's training
// kernels (forward, mean-squared-error gradient, Adam), all FP32 SIMT.
//
// The MLP is 16 -> 64 -> 64 -> 3 with ReLU; the three outputs predict
// log(microseconds) of the PROBE, UNION and HYBRID paths of one query.
// Parameter layout (ABF_PLANNER_PARAMS floats, include/adabool.h):
//   mu[16] sd[16] | W1[64][16] b1[64] | W2[64][64] b2[64] | W3[3][64] b3[3]
// No reference counterpart: the reference runs both of its paths on every
// query (test/adsfilter_q_all.cu:414-452) and has no selection rule.
#include "abf_kernels.cuh"

#include <cmath>

namespace abf {

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
    if (threadIdx.x == 0) {
        n = nd = nl = mx = 0;
        S = Q = Cb = Lg = Sd = Bnd = 0;
        for (int k = 0; k < kFeatThreads / 32; ++k) {
            n += s_u[0][k]; nd += s_u[1][k]; nl += s_u[2][k]; mx = max(mx, s_u[3][k]);
            S += s_d[0][k]; Q += s_d[1][k]; Cb += s_d[2][k]; Lg += s_d[3][k]; Sd += s_d[4][k]; Bnd += s_d[5][k];
        }
        const double nn = n > 0 ? double(n) : 1.0;
        const double mean = S / nn;
        const double var = fmax(Q / nn - mean * mean, 0.0);
        f[0] = float(log1p(double(n)));
        f[1] = float(log1p(S));
        f[2] = float(log1p(double(mx)));
        f[3] = float(log1p(mean));
        f[4] = float(log1p(sqrt(var)));
        f[5] = float(log1p(Cb));
        f[6] = float(1.0 - exp(Lg));
        f[7] = float(log1p(double(nd)));
        f[8] = float(Sd / fmax(S, 1.0));
        f[9] = float(log1p(Bnd));
        f[10] = float(S / double(c.n_postings ? c.n_postings : 1));
        f[11] = float(log1p(double(nl)));
        f[12] = float(double(q) / double(c.n_q ? c.n_q : 1));
        f[13] = float(log1p(double(c.n_q)));
        f[14] = float(double(mx) * inv_ads);
        f[15] = 1.0f;
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

// Fused planner: features -> standardise -> MLP -> cheapest path.
__global__ void __launch_bounds__(kFeatThreads) planner_kernel(IndexView ix, const float* __restrict__ p,
                                                               const uint32_t* terms, const uint64_t* q_off,
                                                               FeatCtx c, float* feat_out, float* pred_out,
                                                               uint8_t* path_out) {
    __shared__ float f[F], xs[F], h1[H], h2[H], y[O];
    for (uint32_t q = blockIdx.x; q < c.n_q; q += gridDim.x) {
        query_features(ix, terms, q_off, q, c, f);
        if (feat_out && threadIdx.x < F) feat_out[uint64_t(q) * F + threadIdx.x] = f[threadIdx.x];
        if (!p) continue;
        if (threadIdx.x < F) {
            const float sd = __ldg(p + kSd + threadIdx.x);
            xs[threadIdx.x] = (f[threadIdx.x] - __ldg(p + kMu + threadIdx.x)) / (sd > 0.0f ? sd : 1.0f);
        }
        __syncthreads();
        mlp_forward_cta(p, xs, h1, h2, y);
        if (threadIdx.x == 0) {
            int best = 0;
            for (int o = 1; o < O; ++o)
                if (y[o] < y[best]) best = o;
            if (pred_out)
                for (int o = 0; o < O; ++o) pred_out[uint64_t(q) * O + o] = y[o];
            if (path_out)
                path_out[q] = uint8_t(best == 0 ? ABF_PATH_PROBE : best == 1 ? ABF_PATH_UNION : ABF_PATH_HYBRID);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(64) mlp_forward_kernel(const float* __restrict__ p, const float* x, uint32_t n,
                                                         float* y_out) {
    __shared__ float xs[F], h1[H], h2[H], y[O];
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x) {
        if (threadIdx.x < F) xs[threadIdx.x] = x[uint64_t(s) * F + threadIdx.x];
        __syncthreads();
        mlp_forward_cta(p, xs, h1, h2, y);
        if (threadIdx.x < O) y_out[uint64_t(s) * O + threadIdx.x] = y[threadIdx.x];
        __syncthreads();
    }
}

__global__ void mask_sum_kernel(const float* mask, uint64_t n, float* out) {
    float s = 0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        s += mask[i] != 0.0f ? 1.0f : 0.0f;
    s = warp_sum(s);
    if (lane() == 0) atomicAdd(out, s);
}

// Gradient of L = sum(mask * (y - t)^2) / sum(mask). 64 threads per CTA,
// thread j owns hidden unit j of both layers; the CTA walks its samples,
// keeps its share of the parameter gradient in registers and adds it to
// d_grad once at the end.
__global__ void __launch_bounds__(64) mlp_grad_kernel(const float* __restrict__ p, const float* x, const float* t,
                                                      const float* mask, uint32_t n, const float* msum, float* g,
                                                      float* loss) {
    __shared__ float xs[F], h1[H], h2[H], y[O], dy[O], dh2[H];
    const int j = threadIdx.x;
    const float inv = 1.0f / fmaxf(*msum, 1.0f);
    float gw1[F], gw2[H], gw3[O];
#pragma unroll
    for (int k = 0; k < F; ++k) gw1[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < H; ++k) gw2[k] = 0.0f;
#pragma unroll
    for (int o = 0; o < O; ++o) gw3[o] = 0.0f;
    float gb1 = 0.0f, gb2 = 0.0f, gb3 = 0.0f, lsum = 0.0f;
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x) {
        if (j < F) xs[j] = x[uint64_t(s) * F + j];
        __syncthreads();
        mlp_forward_cta(p, xs, h1, h2, y);
        if (j < O) {
            const float m = mask[uint64_t(s) * O + j] != 0.0f ? 1.0f : 0.0f;
            const float r = m * (y[j] - t[uint64_t(s) * O + j]);
            dy[j] = 2.0f * r * inv;
            lsum += r * r * inv;
            gb3 += dy[j];
        }
        __syncthreads();
        // layer 3: dW3[o][j] = dy[o] h2[j]; dh2[j] = relu'(h2) sum_o dy[o] W3[o][j]
        float a = 0.0f;
#pragma unroll
        for (int o = 0; o < O; ++o) {
            gw3[o] = fmaf(dy[o], h2[j], gw3[o]);
            a = fmaf(dy[o], __ldg(p + kW3 + o * H + j), a);
        }
        const float d2 = h2[j] > 0.0f ? a : 0.0f;
        dh2[j] = d2;
        gb2 += d2;
        __syncthreads();
        // layer 2: dW2[i][j] = dh2[i] h1[j] (thread j keeps column j);
        // dh1[j] = relu'(h1) sum_i dh2[i] W2[i][j]
        float b = 0.0f;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            gw2[i] = fmaf(dh2[i], h1[j], gw2[i]);
            b = fmaf(dh2[i], __ldg(p + kW2 + i * H + j), b);
        }
        const float d1 = h1[j] > 0.0f ? b : 0.0f;
        gb1 += d1;
#pragma unroll
        for (int k = 0; k < F; ++k) gw1[k] = fmaf(d1, xs[k], gw1[k]);
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < F; ++k) atomicAdd(g + kW1 + j * F + k, gw1[k]);
    atomicAdd(g + kB1 + j, gb1);
#pragma unroll
    for (int i = 0; i < H; ++i) atomicAdd(g + kW2 + i * H + j, gw2[i]);
    atomicAdd(g + kB2 + j, gb2);
#pragma unroll
    for (int o = 0; o < O; ++o) atomicAdd(g + kW3 + o * H + j, gw3[o]);
    if (j < O) {
        atomicAdd(g + kB3 + j, gb3);
        atomicAdd(loss, lsum);
    }
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    for (int i = kW1 + blockIdx.x * blockDim.x + threadIdx.x; i < kNParams; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

int grid_of(uint32_t n, uint32_t cap) { return int(n < cap ? (n ? n : 1) : cap); }

}  // namespace

cudaError_t launch_planner(const IndexView& v, const float* params, const uint32_t* terms, const uint64_t* q_off,
                           uint32_t n_q, uint32_t hybrid_min, uint64_t n_postings, float* feat, float* pred,
                           uint8_t* paths, cudaStream_t s) {
    if (n_q == 0) return cudaSuccess;
    FeatCtx c{hybrid_min, n_postings, n_q};
    planner_kernel<<<grid_of(n_q, 65535u * 4u), kFeatThreads, 0, s>>>(v, params, terms, q_off, c, feat, pred, paths);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const float* p, const float* x, uint32_t n, float* y, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    mlp_forward_kernel<<<grid_of(n, 148u * 16u), 64, 0, s>>>(p, x, n, y);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const float* p, const float* x, const float* t, const float* mask, uint32_t n, float* g,
                            float* loss2, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(g, 0, sizeof(float) * kNParams, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(loss2, 0, 2 * sizeof(float), s);
    if (e != cudaSuccess || n == 0) return e;
    mask_sum_kernel<<<grid_of((n * O + 255) / 256, 256u), 256, 0, s>>>(mask, uint64_t(n) * O, loss2 + 1);
    mlp_grad_kernel<<<grid_of(n, 148u * 8u), 64, 0, s>>>(p, x, t, mask, n, loss2 + 1, g, loss2);
    count_launch(2);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* p, const float* g, float* m, float* v, uint32_t step, float lr, float b1, float b2,
                        float eps, cudaStream_t s) {
    const float c1 = 1.0f - std::pow(b1, float(step ? step : 1));
    const float c2 = 1.0f - std::pow(b2, float(step ? step : 1));
    adam_kernel<<<(kNParams + 255) / 256, 256, 0, s>>>(p, g, m, v, lr, b1, b2, eps, c1, c2);
    count_launch();
    return cudaGetLastError();
}

}  // namespace abf
