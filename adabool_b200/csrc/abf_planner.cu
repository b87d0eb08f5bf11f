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
#include "abf_planner_dev.cuh"

#include <cmath>

namespace abf {

namespace {

using namespace plan_dev;

// Fused planner: features -> standardise -> MLP -> cheapest path.
__global__ void __launch_bounds__(kFeatThreads) planner_kernel(IndexView ix, const float* __restrict__ p,
                                                               const uint32_t* terms, const uint64_t* q_off,
                                                               FeatCtx c, float* feat_out, float* pred_out,
                                                               uint8_t* path_out) {
    __shared__ PlannerSmem sm;
    for (uint32_t q = blockIdx.x; q < c.n_q; q += gridDim.x) {
        if (!p) {
            query_features(ix, terms, q_off, q, c, sm.f);
            if (feat_out && threadIdx.x < F) feat_out[uint64_t(q) * F + threadIdx.x] = sm.f[threadIdx.x];
            continue;
        }
        const uint32_t path = planner_path(ix, p, terms, q_off, q, c, sm);
        if (feat_out && threadIdx.x < F) feat_out[uint64_t(q) * F + threadIdx.x] = sm.f[threadIdx.x];
        if (threadIdx.x == 0) {
            if (pred_out)
                for (int o = 0; o < O; ++o) pred_out[uint64_t(q) * O + o] = sm.y[o];
            if (path_out) path_out[q] = uint8_t(path);
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
