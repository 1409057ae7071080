// amx_selector.cu -- the learned format selector's network: a 16 -> 64 -> 64 -> K FP32 MLP
// (ReLU hidden layers, softmax output) with hand-written inference and training kernels.
//
// The network only chooses storage formats and widths for the intermediate columns of an
// operator chain; it never touches the integer arithmetic, so the chain's results are the same
// whatever it picks.  The reference has no counterpart (its formats are compile-time choices of
// each benchmark, src/main.cu:300-340).
//
// Parameter layout (floats, contiguous): W1[64][16] b1[64] W2[64][64] b2[64] W3[K][64] b3[K].
//
//   mlp_forward_kernel  one warp per sample, probabilities out;
//   mlp_train_kernel    one CTA runs a whole mini-batch deterministically: per sample a forward
//                       pass, softmax cross-entropy and the backward pass, with every gradient
//                       entry owned by one thread (no atomics, the same sums in the same order on
//                       every run), then one Adam step.
#include <cmath>

#include "amx_dispatch.h"

namespace amx {

constexpr int kMlpIn = 16;
constexpr int kMlpH = 64;
constexpr int kMlpMaxK = 8;
constexpr int kMlpTrainThreads = 256;

__host__ __device__ constexpr int mlp_params(int K) { return kMlpH * kMlpIn + kMlpH + kMlpH * kMlpH + kMlpH + K * kMlpH + K; }

struct MlpView {
    const float *W1, *b1, *W2, *b2, *W3, *b3;
};

__device__ __forceinline__ MlpView mlp_view(const float* p, int K)
{
    MlpView v;
    v.W1 = p;
    v.b1 = v.W1 + kMlpH * kMlpIn;
    v.W2 = v.b1 + kMlpH;
    v.b2 = v.W2 + kMlpH * kMlpH;
    v.W3 = v.b2 + kMlpH;
    v.b3 = v.W3 + K * kMlpH;
    (void)K;
    return v;
}

__global__ void __launch_bounds__(256) mlp_forward_kernel(const float* __restrict__ params, int K,
                                                          const float* __restrict__ x, uint32_t batch,
                                                          float* __restrict__ probs)
{
    __shared__ float h1s[8][kMlpH];
    __shared__ float h2s[8][kMlpH];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const MlpView P = mlp_view(params, K);
    for (uint32_t s = blockIdx.x * 8 + w; s < batch; s += gridDim.x * 8) {
        const float* xs = x + (size_t)s * kMlpIn;
        for (int j = lane; j < kMlpH; j += 32) {
            float a = P.b1[j];
            for (int i = 0; i < kMlpIn; i++) a += P.W1[j * kMlpIn + i] * xs[i];
            h1s[w][j] = a > 0.f ? a : 0.f;
        }
        __syncwarp();
        for (int j = lane; j < kMlpH; j += 32) {
            float a = P.b2[j];
            for (int i = 0; i < kMlpH; i++) a += P.W2[j * kMlpH + i] * h1s[w][i];
            h2s[w][j] = a > 0.f ? a : 0.f;
        }
        __syncwarp();
        float z = -INFINITY;
        if ((int)lane < K) {
            z = P.b3[lane];
            for (int i = 0; i < kMlpH; i++) z += P.W3[lane * kMlpH + i] * h2s[w][i];
        }
        float mx = z;
        for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        const float e = (int)lane < K ? expf(z - mx) : 0.f;
        float sum = e;
        for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if ((int)lane < K) probs[(size_t)s * K + lane] = e / sum;
        __syncwarp();
    }
}

// One mini-batch of softmax cross-entropy and one Adam step (beta1 0.9, beta2 0.999, eps 1e-8).
// adam = [m | v], 2 * mlp_params(K) floats; step counts from 1.
__global__ void __launch_bounds__(kMlpTrainThreads) mlp_train_kernel(float* __restrict__ params,
                                                                     float* __restrict__ adam, uint32_t step, int K,
                                                                     const float* __restrict__ x,
                                                                     const uint32_t* __restrict__ labels,
                                                                     uint32_t batch, float lr, float* loss_out)
{
    extern __shared__ float sm[];
    const int NP = mlp_params(K);
    float* p = sm;        // parameters
    float* g = sm + NP;   // gradients
    float* act = g + NP;  // x[16] h1[64] h2[64] z/p[8] dz[8] dh2[64] dh1[64]
    float* xs = act;
    float* h1 = xs + kMlpIn;
    float* h2 = h1 + kMlpH;
    float* pr = h2 + kMlpH;
    float* dz = pr + kMlpMaxK;
    float* dh2 = dz + kMlpMaxK;
    float* dh1 = dh2 + kMlpH;
    __shared__ float s_loss;
    const int t = threadIdx.x;
    for (int i = t; i < NP; i += kMlpTrainThreads) {
        p[i] = params[i];
        g[i] = 0.f;
    }
    if (t == 0) s_loss = 0.f;
    __syncthreads();
    float* W1 = p;
    float* b1 = W1 + kMlpH * kMlpIn;
    float* W2 = b1 + kMlpH;
    float* b2 = W2 + kMlpH * kMlpH;
    float* W3 = b2 + kMlpH;
    float* b3 = W3 + K * kMlpH;
    float* gW1 = g;
    float* gb1 = gW1 + kMlpH * kMlpIn;
    float* gW2 = gb1 + kMlpH;
    float* gb2 = gW2 + kMlpH * kMlpH;
    float* gW3 = gb2 + kMlpH;
    float* gb3 = gW3 + K * kMlpH;

    for (uint32_t s = 0; s < batch; s++) {
        if (t < kMlpIn) xs[t] = x[(size_t)s * kMlpIn + t];
        __syncthreads();
        if (t < kMlpH) {
            float a = b1[t];
            for (int i = 0; i < kMlpIn; i++) a += W1[t * kMlpIn + i] * xs[i];
            h1[t] = a > 0.f ? a : 0.f;
        }
        __syncthreads();
        if (t < kMlpH) {
            float a = b2[t];
            for (int i = 0; i < kMlpH; i++) a += W2[t * kMlpH + i] * h1[i];
            h2[t] = a > 0.f ? a : 0.f;
        }
        __syncthreads();
        if (t < K) {
            float z = b3[t];
            for (int i = 0; i < kMlpH; i++) z += W3[t * kMlpH + i] * h2[i];
            pr[t] = z;
        }
        __syncthreads();
        if (t == 0) {
            float mx = pr[0];
            for (int k = 1; k < K; k++) mx = fmaxf(mx, pr[k]);
            float sum = 0.f;
            for (int k = 0; k < K; k++) {
                pr[k] = expf(pr[k] - mx);
                sum += pr[k];
            }
            const uint32_t y = labels[s];
            for (int k = 0; k < K; k++) {
                pr[k] /= sum;
                dz[k] = pr[k] - ((uint32_t)k == y ? 1.f : 0.f);
            }
            s_loss -= logf(fmaxf(pr[y], 1e-30f));
        }
        __syncthreads();
        for (int i = t; i < K * kMlpH; i += kMlpTrainThreads) gW3[i] += dz[i / kMlpH] * h2[i % kMlpH];
        if (t < K) gb3[t] += dz[t];
        if (t < kMlpH) {
            float a = 0.f;
            for (int k = 0; k < K; k++) a += W3[k * kMlpH + t] * dz[k];
            dh2[t] = h2[t] > 0.f ? a : 0.f;
        }
        __syncthreads();
        for (int i = t; i < kMlpH * kMlpH; i += kMlpTrainThreads) gW2[i] += dh2[i / kMlpH] * h1[i % kMlpH];
        if (t < kMlpH) {
            gb2[t] += dh2[t];
            float a = 0.f;
            for (int j = 0; j < kMlpH; j++) a += W2[j * kMlpH + t] * dh2[j];
            dh1[t] = h1[t] > 0.f ? a : 0.f;
        }
        __syncthreads();
        for (int i = t; i < kMlpH * kMlpIn; i += kMlpTrainThreads) gW1[i] += dh1[i / kMlpIn] * xs[i % kMlpIn];
        if (t < kMlpH) gb1[t] += dh1[t];
        __syncthreads();
    }
    // Adam on the mean gradient
    const float inv = batch ? 1.f / (float)batch : 0.f;
    const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
    float* m = adam;
    float* v = adam + NP;
    for (int i = t; i < NP; i += kMlpTrainThreads) {
        const float gr = g[i] * inv;
        const float mi = 0.9f * m[i] + 0.1f * gr;
        const float vi = 0.999f * v[i] + 0.001f * gr * gr;
        m[i] = mi;
        v[i] = vi;
        params[i] = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    }
    if (t == 0 && loss_out) *loss_out = s_loss * inv;
}

}  // namespace amx

using namespace amx;

extern "C" {

uint32_t amx_mlp_param_count(uint32_t classes)
{
    return (classes >= 2 && classes <= (uint32_t)kMlpMaxK) ? (uint32_t)mlp_params((int)classes) : 0;
}

amx_status amx_mlp_forward(const float* d_params, uint32_t classes, const float* d_x, uint32_t batch, float* d_probs,
                           void* stream)
{
    if (classes < 2 || classes > (uint32_t)kMlpMaxK) return fail(AMX_ERR_INVALID_ARG, "mlp: %u classes", classes);
    if (!batch) return AMX_OK;
    if (!d_params || !d_x || !d_probs) return fail(AMX_ERR_INVALID_ARG, "mlp_forward: null pointer");
    const uint32_t blocks = (batch + 7) / 8 < 1024 ? (batch + 7) / 8 : 1024;
    mlp_forward_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d_params, (int)classes, d_x, batch, d_probs);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AMX_OK : cuda_fail(e, "mlp_forward launch");
}

amx_status amx_mlp_train_step(float* d_params, float* d_adam, uint32_t step, uint32_t classes, const float* d_x,
                              const uint32_t* d_labels, uint32_t batch, float lr, float* d_loss, void* stream)
{
    if (classes < 2 || classes > (uint32_t)kMlpMaxK) return fail(AMX_ERR_INVALID_ARG, "mlp: %u classes", classes);
    if (!d_params || !d_adam || (batch && (!d_x || !d_labels)))
        return fail(AMX_ERR_INVALID_ARG, "mlp_train_step: null pointer");
    if (step < 1) return fail(AMX_ERR_INVALID_ARG, "mlp_train_step: steps count from 1");
    const size_t smem = (2 * (size_t)mlp_params((int)classes) + kMlpIn + 4 * kMlpH + 2 * kMlpMaxK) * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "mlp_train_step: shared memory attribute");
    mlp_train_kernel<<<1, kMlpTrainThreads, smem, (cudaStream_t)stream>>>(d_params, d_adam, step, (int)classes, d_x,
                                                                         d_labels, batch, lr, d_loss);
    e = cudaGetLastError();
    return e == cudaSuccess ? AMX_OK : cuda_fail(e, "mlp_train_step launch");
}

}  // extern "C"
