// mlp.cu -- the learned launch tuner's network: a small MLP trained and run
// on the GPU by these kernels (no counterpart in the reference).
//
// Network: x[9] -> 32 ReLU -> 32 ReLU -> y[2], fp32.  The input is a batch's
// features (log2 size, entropy, longest code, level-2 byte fraction) and a
// launch shape (encoder region size, histogram / encoder / decoder CTAs per
// SM, decoder tile size), normalised by the host; the outputs are the predicted log times of
// the batched compress and decompress.  Parameters are one flat fp32 array:
// W1[32][9] b1[32] W2[32][32] b2[32] W3[2][32] b3[2].
//
// Kernels: forward (one thread per sample, parameters staged in shared
// memory); loss + gradient (one thread per sample, the per-sample gradient
// reduced over the warp with shuffles, then one atomic per parameter per
// warp); Adam.  Targets that are NaN are not measured and carry no loss.
#include <cuda_runtime.h>

#include <cmath>

#include "hgap_internal.h"

namespace hgap {
namespace {

constexpr int kIn = HGAP_MLP_IN, kHid = HGAP_MLP_HIDDEN, kOut = HGAP_MLP_OUT;
constexpr int kW1 = 0, kB1 = kW1 + kHid * kIn, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid;
constexpr int kW3 = kB2 + kHid, kB3 = kW3 + kOut * kHid, kParams = kB3 + kOut;
static_assert(kParams == HGAP_MLP_PARAMS, "parameter layout");
constexpr int kThreads = 256;

__device__ __forceinline__ void load_params(const float* __restrict__ p, float* s) {
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) s[i] = p[i];
    __syncthreads();
}

// h1, h2 post-activation; returns y.  Outer loops stay rolled: the network
// is tiny and a full unroll only trades registers for spills.
__device__ __forceinline__ void forward_one(const float* s, const float* x, float* h1, float* h2, float* y) {
#pragma unroll 1
    for (int j = 0; j < kHid; ++j) {
        float a = s[kB1 + j];
#pragma unroll
        for (int i = 0; i < kIn; ++i) a = fmaf(s[kW1 + j * kIn + i], x[i], a);
        h1[j] = a > 0.f ? a : 0.f;
    }
#pragma unroll 1
    for (int k = 0; k < kHid; ++k) {
        float a = s[kB2 + k];
#pragma unroll 8
        for (int j = 0; j < kHid; ++j) a = fmaf(s[kW2 + k * kHid + j], h1[j], a);
        h2[k] = a > 0.f ? a : 0.f;
    }
#pragma unroll
    for (int o = 0; o < kOut; ++o) {
        float a = s[kB3 + o];
#pragma unroll 8
        for (int k = 0; k < kHid; ++k) a = fmaf(s[kW3 + o * kHid + k], h2[k], a);
        y[o] = a;
    }
}

__global__ void __launch_bounds__(kThreads) mlp_forward_kernel(const float* __restrict__ params,
                                                               const float* __restrict__ X, uint32_t n,
                                                               float* __restrict__ Y) {
    __shared__ float s[kParams];
    load_params(params, s);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        float x[kIn], h1[kHid], h2[kHid], y[kOut];
#pragma unroll
        for (int i = 0; i < kIn; ++i) x[i] = X[(uint64_t)r * kIn + i];
        forward_one(s, x, h1, h2, y);
#pragma unroll
        for (int o = 0; o < kOut; ++o) Y[(uint64_t)r * kOut + o] = y[o];
    }
}

// Adds the warp's sum of v to *dst (lane 0).
__device__ __forceinline__ void warp_add(float v, float* dst) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0 && v != 0.f) atomicAdd(dst, v);
}

// loss = scale * sum over samples and measured outputs of (y - t)^2 / 2;
// grad += d loss / d params.  grad and loss are zeroed by the caller.
__global__ void __launch_bounds__(kThreads) mlp_grad_kernel(const float* __restrict__ params,
                                                            const float* __restrict__ X,
                                                            const float* __restrict__ T, uint32_t n,
                                                            float scale, float* __restrict__ grad,
                                                            float* __restrict__ loss) {
    __shared__ float s[kParams];
    load_params(params, s);
    // every lane of a warp runs every sample slot (shuffles need all lanes)
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounds = (n + stride - 1) / stride;
    for (uint32_t k = 0; k < rounds; ++k) {
        const uint32_t r = k * stride + blockIdx.x * blockDim.x + threadIdx.x;
        const bool have = r < n;
        float x[kIn], h1[kHid], h2[kHid], y[kOut], gy[kOut];
#pragma unroll
        for (int i = 0; i < kIn; ++i) x[i] = have ? X[(uint64_t)r * kIn + i] : 0.f;
        forward_one(s, x, h1, h2, y);
        float l = 0.f;
#pragma unroll
        for (int o = 0; o < kOut; ++o) {
            const float t = have ? T[(uint64_t)r * kOut + o] : 0.f;
            const bool valid = have && !isnan(t);
            const float d = valid ? y[o] - t : 0.f;
            gy[o] = d * scale;
            l += 0.5f * d * d * scale;
        }
        warp_add(l, loss);
        // output layer
        float gh2[kHid];
#pragma unroll
        for (int kk = 0; kk < kHid; ++kk) gh2[kk] = 0.f;
#pragma unroll
        for (int o = 0; o < kOut; ++o) {
            warp_add(gy[o], grad + kB3 + o);
#pragma unroll
            for (int kk = 0; kk < kHid; ++kk) {
                warp_add(gy[o] * h2[kk], grad + kW3 + o * kHid + kk);
                gh2[kk] = fmaf(gy[o], s[kW3 + o * kHid + kk], gh2[kk]);
            }
        }
        // second hidden layer
        float gh1[kHid];
#pragma unroll
        for (int j = 0; j < kHid; ++j) gh1[j] = 0.f;
        for (int kk = 0; kk < kHid; ++kk) {
            const float g = h2[kk] > 0.f ? gh2[kk] : 0.f;
            warp_add(g, grad + kB2 + kk);
#pragma unroll
            for (int j = 0; j < kHid; ++j) {
                warp_add(g * h1[j], grad + kW2 + kk * kHid + j);
                gh1[j] = fmaf(g, s[kW2 + kk * kHid + j], gh1[j]);
            }
        }
        // first hidden layer
        for (int j = 0; j < kHid; ++j) {
            const float g = h1[j] > 0.f ? gh1[j] : 0.f;
            warp_add(g, grad + kB1 + j);
#pragma unroll
            for (int i = 0; i < kIn; ++i) warp_add(g * x[i], grad + kW1 + j * kIn + i);
        }
    }
}

// Adam on the gradient plus an L2 term (weight_decay * p).
__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, float lr, float b1, float b2, float eps, float wd,
                                float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float gi = fmaf(wd, p[i], g[i]);
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline hgap_status cuda_status(cudaError_t e) { return e == cudaSuccess ? HGAP_OK : HGAP_ERR_CUDA; }

unsigned grid_for(uint32_t n) {
    const uint32_t b = (n + kThreads - 1) / kThreads;
    return b ? (b > 1024 ? 1024 : b) : 1;
}

}  // namespace
}  // namespace hgap

using namespace hgap;

extern "C" {

hgap_status hgap_mlp_forward(const float* d_params, const float* d_x, uint32_t n, float* d_y,
                             hgap_stream_t stream) {
    if (n == 0) return HGAP_OK;
    if (!d_params || !d_x || !d_y) return HGAP_ERR_INVALID_ARG;
    mlp_forward_kernel<<<grid_for(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_params, d_x, n,
                                                                                              d_y);
    return cuda_status(cudaGetLastError());
}

hgap_status hgap_mlp_loss_grad(const float* d_params, const float* d_x, const float* d_target, uint32_t n,
                               float scale, float* d_grad, float* d_loss, hgap_stream_t stream) {
    if (!d_params || !d_x || !d_target || !d_grad || !d_loss) return HGAP_ERR_INVALID_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(d_grad, 0, sizeof(float) * kParams, st) != cudaSuccess) return HGAP_ERR_CUDA;
    if (cudaMemsetAsync(d_loss, 0, sizeof(float), st) != cudaSuccess) return HGAP_ERR_CUDA;
    if (n == 0) return HGAP_OK;
    mlp_grad_kernel<<<grid_for(n), kThreads, 0, st>>>(d_params, d_x, d_target, n, scale, d_grad, d_loss);
    return cuda_status(cudaGetLastError());
}

hgap_status hgap_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, uint32_t step,
                          float lr, float beta1, float beta2, float eps, float weight_decay, hgap_stream_t stream) {
    if (!d_params || !d_grad || !d_m || !d_v || step == 0) return HGAP_ERR_INVALID_ARG;
    const float c1 = 1.f - (float)std::pow((double)beta1, (double)step);
    const float c2 = 1.f - (float)std::pow((double)beta2, (double)step);
    mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        d_params, d_grad, d_m, d_v, lr, beta1, beta2, eps, weight_decay, c1, c2);
    return cuda_status(cudaGetLastError());
}

}  // extern "C"
