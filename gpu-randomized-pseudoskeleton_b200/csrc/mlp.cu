// Rank / sample-count predictor: an 8 -> 64 -> 64 -> 1 MLP with GELU, FP32, trained and run
// by the kernels in this file (forward, backward with weight-gradient reduction, Adam).
//
// Layout (row-major, one contiguous parameter vector of kMlpParams floats):
//   W1 [64 x 8], b1 [64], W2 [64 x 64], b2 [64], W3 [1 x 64], b3 [1]
// Inputs are standardised by the caller (x' = (x - mean) / std); the output is log2 of the
// sample count. GELU is the tanh form 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
// (Hendrycks & Gimpel 2016), evaluated with tanhf.
//
// The network is tiny (4.8 k parameters) and the batches are thousands of blocks, so one
// thread owns one sample through all three layers with the weights staged in shared memory;
// the backward pass sums each weight gradient over the warp with shuffles, accumulates the
// warps of a CTA in shared memory and adds the CTA total to the global gradient.
#include <cmath>

#include "pskel_internal.cuh"

namespace pskel {

constexpr int kIn = 8, kH = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kIn, kOffW2 = kOffB1 + kH,
              kOffB2 = kOffW2 + kH * kH, kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH,
              kMlpParams = kOffB3 + 1;

__device__ __forceinline__ float gelu_f(float x, float *dgelu) {
    const float c = 0.7978845608028654f;  // sqrt(2/pi)
    const float u = c * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    if (dgelu) {
        const float du = c * (1.0f + 3.0f * 0.044715f * x * x);
        *dgelu = 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * du;
    }
    return 0.5f * x * (1.0f + t);
}

__global__ void __launch_bounds__(128) mlp_forward_kernel(const float *__restrict__ params,
                                                          const float *__restrict__ x, int n,
                                                          float *__restrict__ y) {
    __shared__ float w[kMlpParams];
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) w[i] = params[i];
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float in[kIn], h1[kH];
#pragma unroll
    for (int k = 0; k < kIn; ++k) in[k] = x[(size_t)s * kIn + k];
#pragma unroll 4
    for (int j = 0; j < kH; ++j) {
        float a = w[kOffB1 + j];
#pragma unroll
        for (int k = 0; k < kIn; ++k) a = fmaf(w[kOffW1 + j * kIn + k], in[k], a);
        h1[j] = gelu_f(a, nullptr);
    }
    float out = w[kOffB3];
    for (int j = 0; j < kH; ++j) {
        float a = w[kOffB2 + j];
#pragma unroll 8
        for (int k = 0; k < kH; ++k) a = fmaf(w[kOffW2 + j * kH + k], h1[k], a);
        out = fmaf(w[kOffW3 + j], gelu_f(a, nullptr), out);
    }
    y[s] = out;
}

// Sum over the warp, then one shared-memory atomic per warp.
__device__ __forceinline__ void warp_add(float v, float *dst) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(dst, v);
}

// Mean-squared-error gradient of a batch: grad (kMlpParams, zeroed by the caller) receives
// d/dparams of (1/n) sum (y_s - t_s)^2 and loss[0] the summed squared error. Threads past the
// end of the batch run the same loops with a zero error so that every warp reduction is full.
__global__ void __launch_bounds__(128) mlp_backward_kernel(const float *__restrict__ params,
                                                           const float *__restrict__ x,
                                                           const float *__restrict__ target,
                                                           int n, float *__restrict__ grad,
                                                           float *__restrict__ loss) {
    __shared__ float w[kMlpParams];
    __shared__ float g[kMlpParams];
    __shared__ float s_loss;
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
        w[i] = params[i];
        g[i] = 0.0f;
    }
    if (threadIdx.x == 0) s_loss = 0.0f;
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = s < n;
    float in[kIn], h1[kH], d1[kH], a2[kH];
#pragma unroll
    for (int k = 0; k < kIn; ++k) in[k] = live ? x[(size_t)s * kIn + k] : 0.0f;
    for (int j = 0; j < kH; ++j) {
        float a = w[kOffB1 + j];
#pragma unroll
        for (int k = 0; k < kIn; ++k) a = fmaf(w[kOffW1 + j * kIn + k], in[k], a);
        h1[j] = gelu_f(a, &d1[j]);
    }
    float out = w[kOffB3];
    for (int j = 0; j < kH; ++j) {
        float a = w[kOffB2 + j];
        for (int k = 0; k < kH; ++k) a = fmaf(w[kOffW2 + j * kH + k], h1[k], a);
        a2[j] = a;
        out = fmaf(w[kOffW3 + j], gelu_f(a, nullptr), out);
    }
    const float err = live ? out - target[s] : 0.0f;
    warp_add(err * err, &s_loss);
    const float dy = 2.0f * err / (float)n;
    warp_add(dy, &g[kOffB3]);
    float dh1[kH];
#pragma unroll 8
    for (int k = 0; k < kH; ++k) dh1[k] = 0.0f;
    for (int j = 0; j < kH; ++j) {
        float dg;
        const float h2 = gelu_f(a2[j], &dg);
        warp_add(dy * h2, &g[kOffW3 + j]);
        const float da2 = dy * w[kOffW3 + j] * dg;
        warp_add(da2, &g[kOffB2 + j]);
        for (int k = 0; k < kH; ++k) {
            warp_add(da2 * h1[k], &g[kOffW2 + j * kH + k]);
            dh1[k] = fmaf(da2, w[kOffW2 + j * kH + k], dh1[k]);
        }
    }
    for (int j = 0; j < kH; ++j) {
        const float da1 = dh1[j] * d1[j];
        warp_add(da1, &g[kOffB1 + j]);
#pragma unroll
        for (int k = 0; k < kIn; ++k) warp_add(da1 * in[k], &g[kOffW1 + j * kIn + k]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) atomicAdd(&grad[i], g[i]);
    if (threadIdx.x == 0) atomicAdd(loss, s_loss);
}

// Adam (Kingma & Ba 2015) with bias correction; step t >= 1.
__global__ void mlp_adam_kernel(float *__restrict__ params, const float *__restrict__ grad,
                                float *__restrict__ m, float *__restrict__ v, int t, float lr,
                                float beta1, float beta2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const float gi = grad[i];
    const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.0f - powf(beta1, (float)t));
    const float vh = vi / (1.0f - powf(beta2, (float)t));
    params[i] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace pskel

using namespace pskel;

extern "C" int pskel_mlp_num_params(void) { return kMlpParams; }

extern "C" int pskel_mlp_forward(const float *params_dev, const float *x_dev, int n, float *y_dev,
                                 void *stream) {
    if (!params_dev || (n > 0 && (!x_dev || !y_dev)) || n < 0) {
        set_error(PSKEL_ERR_ARG, "mlp_forward: bad arguments");
        return PSKEL_ERR_ARG;
    }
    if (n == 0) return PSKEL_OK;
    mlp_forward_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(params_dev, x_dev, n, y_dev);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

extern "C" int pskel_mlp_grad(const float *params_dev, const float *x_dev, const float *t_dev,
                              int n, float *grad_dev, float *loss_dev, void *stream) {
    if (!params_dev || !grad_dev || !loss_dev || n <= 0 || !x_dev || !t_dev) {
        set_error(PSKEL_ERR_ARG, "mlp_grad: bad arguments");
        return PSKEL_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    PSKEL_CUDA(cudaMemsetAsync(grad_dev, 0, sizeof(float) * kMlpParams, s));
    PSKEL_CUDA(cudaMemsetAsync(loss_dev, 0, sizeof(float), s));
    mlp_backward_kernel<<<(n + 127) / 128, 128, 0, s>>>(params_dev, x_dev, t_dev, n, grad_dev, loss_dev);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

extern "C" int pskel_mlp_adam(float *params_dev, const float *grad_dev, float *m_dev, float *v_dev,
                              int t, float lr, float beta1, float beta2, float eps, void *stream) {
    if (!params_dev || !grad_dev || !m_dev || !v_dev || t < 1) {
        set_error(PSKEL_ERR_ARG, "mlp_adam: bad arguments");
        return PSKEL_ERR_ARG;
    }
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        params_dev, grad_dev, m_dev, v_dev, t, lr, beta1, beta2, eps);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}
