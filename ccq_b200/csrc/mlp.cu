// Warm-start network: a small multilayer perceptron over per-amplitude features,
// trained and evaluated on the GPU with these kernels (no library calls).
//
//   y = w3 . tanh(W2 tanh(W1 x + b1) + b2) + b3,   x in R^F (F <= MLP_MAXF), hidden width H = MLP_H
//
// Parameters live in one float array (FP32; accumulation in FP32):
//   W1[H][F] | b1[H] | W2[H][H] | b2[H] | w3[H] | b3
// One thread evaluates one sample with the parameters staged in shared memory.
// The backward kernel recomputes the forward pass, forms the gradient of the
// mean-squared loss 1/N sum (y - t)^2 and reduces it per block in shared memory
// before one global atomic per parameter and block.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ccq_b200.h"

namespace {

constexpr int H = CCQ_B200_MLP_HIDDEN;
constexpr int MAXF = CCQ_B200_MLP_MAXF;

__host__ __device__ constexpr int nparams(int F) { return H * F + H + H * H + H + H + 1; }

__global__ void __launch_bounds__(128) mlp_forward_kernel(const float *__restrict__ P, int F,
                                                          const float *__restrict__ X, long long N,
                                                          float *__restrict__ Y) {
    extern __shared__ float sp[];
    const int np = nparams(F);
    for (int i = threadIdx.x; i < np; i += blockDim.x) sp[i] = P[i];
    __syncthreads();
    const float *W1 = sp, *b1 = W1 + H * F, *W2 = b1 + H, *b2 = W2 + H * H, *w3 = b2 + H, *b3 = w3 + H;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
        float x[MAXF];
#pragma unroll
        for (int f = 0; f < MAXF; ++f) x[f] = f < F ? X[s * F + f] : 0.f;
        float h1[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            float z = b1[j];
#pragma unroll
            for (int f = 0; f < MAXF; ++f)
                if (f < F) z += W1[j * F + f] * x[f];
            h1[j] = tanhf(z);
        }
        float y = b3[0];
#pragma unroll 4
        for (int k = 0; k < H; ++k) {
            float z = b2[k];
#pragma unroll
            for (int j = 0; j < H; ++j) z += W2[k * H + j] * h1[j];
            y += w3[k] * tanhf(z);
        }
        Y[s] = y;
    }
}

__global__ void __launch_bounds__(128) mlp_backward_kernel(const float *__restrict__ P, int F,
                                                           const float *__restrict__ X,
                                                           const float *__restrict__ T, long long N,
                                                           float *__restrict__ G, float *__restrict__ loss) {
    extern __shared__ float sm[];
    const int np = nparams(F);
    float *sp = sm, *sg = sm + np;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        sp[i] = P[i];
        sg[i] = 0.f;
    }
    __shared__ float sloss;
    if (threadIdx.x == 0) sloss = 0.f;
    __syncthreads();
    const float *W1 = sp, *b1 = W1 + H * F, *W2 = b1 + H, *b2 = W2 + H * H, *w3 = b2 + H, *b3 = w3 + H;
    float *gW1 = sg, *gb1 = gW1 + H * F, *gW2 = gb1 + H, *gb2 = gW2 + H * H, *gw3 = gb2 + H, *gb3 = gw3 + H;
    const float inv = 1.f / (float)N;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
        float x[MAXF];
#pragma unroll
        for (int f = 0; f < MAXF; ++f) x[f] = f < F ? X[s * F + f] : 0.f;
        float h1[H], h2[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            float z = b1[j];
#pragma unroll
            for (int f = 0; f < MAXF; ++f)
                if (f < F) z += W1[j * F + f] * x[f];
            h1[j] = tanhf(z);
        }
        float y = b3[0];
#pragma unroll
        for (int k = 0; k < H; ++k) {
            float z = b2[k];
#pragma unroll
            for (int j = 0; j < H; ++j) z += W2[k * H + j] * h1[j];
            h2[k] = tanhf(z);
            y += w3[k] * h2[k];
        }
        const float r = y - T[s];
        atomicAdd(&sloss, r * r * inv);
        const float g = 2.f * r * inv;
        atomicAdd(gb3, g);
        float g1[H];
#pragma unroll
        for (int j = 0; j < H; ++j) g1[j] = 0.f;
#pragma unroll
        for (int k = 0; k < H; ++k) {
            atomicAdd(gw3 + k, g * h2[k]);
            const float g2 = g * w3[k] * (1.f - h2[k] * h2[k]);
            atomicAdd(gb2 + k, g2);
#pragma unroll
            for (int j = 0; j < H; ++j) {
                atomicAdd(gW2 + k * H + j, g2 * h1[j]);
                g1[j] += W2[k * H + j] * g2;
            }
        }
#pragma unroll
        for (int j = 0; j < H; ++j) {
            const float gz = g1[j] * (1.f - h1[j] * h1[j]);
            atomicAdd(gb1 + j, gz);
#pragma unroll
            for (int f = 0; f < MAXF; ++f)
                if (f < F) atomicAdd(gW1 + j * F + f, gz * x[f]);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += blockDim.x)
        if (sg[i] != 0.f) atomicAdd(G + i, sg[i]);
    if (threadIdx.x == 0) atomicAdd(loss, sloss);
}

// Adam step on every parameter (bias-corrected moments, step t >= 1)
__global__ void adam_kernel(float *P, const float *G, float *m, float *v, int np, float lr, float b1, float b2,
                            float eps, int t) {
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const float g = G[i];
        m[i] = b1 * m[i] + (1.f - b1) * g;
        v[i] = b2 * v[i] + (1.f - b2) * g * g;
        P[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
    }
}

int grid_for(long long n) {
    long long b = (n + 127) / 128;
    if (b > 148 * 8) b = 148 * 8;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" int ccq_b200_mlp_params(int64_t nfeat) {
    if (nfeat < 1 || nfeat > MAXF) return CCQ_B200_EINVAL;
    return nparams((int)nfeat);
}

extern "C" int ccq_b200_mlp_forward(const float *params, int64_t nfeat, const float *x, int64_t n, float *y,
                                    void *stream) {
    if (!params || !x || !y || nfeat < 1 || nfeat > MAXF || n < 0) return CCQ_B200_EINVAL;
    if (n == 0) return 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t sh = sizeof(float) * nparams((int)nfeat);
    mlp_forward_kernel<<<grid_for(n), 128, sh, s>>>(params, (int)nfeat, x, n, y);
    return cudaGetLastError() == cudaSuccess ? 0 : CCQ_B200_ECUDA;
}

extern "C" int ccq_b200_mlp_grad(const float *params, int64_t nfeat, const float *x, const float *target, int64_t n,
                                 float *grad, float *loss, void *stream) {
    if (!params || !x || !target || !grad || !loss || nfeat < 1 || nfeat > MAXF || n < 1) return CCQ_B200_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int np = nparams((int)nfeat);
    if (cudaMemsetAsync(grad, 0, sizeof(float) * np, s) != cudaSuccess) return CCQ_B200_ECUDA;
    if (cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) return CCQ_B200_ECUDA;
    const size_t sh = sizeof(float) * 2 * np;
    mlp_backward_kernel<<<grid_for(n), 128, sh, s>>>(params, (int)nfeat, x, target, n, grad, loss);
    return cudaGetLastError() == cudaSuccess ? 0 : CCQ_B200_ECUDA;
}

extern "C" int ccq_b200_mlp_adam(float *params, const float *grad, float *m, float *v, int64_t nparam, double lr,
                                 int64_t step, void *stream) {
    if (!params || !grad || !m || !v || nparam < 1 || step < 1) return CCQ_B200_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    adam_kernel<<<grid_for(nparam), 128, 0, s>>>(params, grad, m, v, (int)nparam, (float)lr, 0.9f, 0.999f, 1e-8f,
                                                 (int)step);
    return cudaGetLastError() == cudaSuccess ? 0 : CCQ_B200_ECUDA;
}
