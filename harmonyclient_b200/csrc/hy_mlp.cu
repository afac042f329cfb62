// The learned probe predictor: a small MLP that reads a query's sorted
// centroid distances and predicts how many lists it needs (its "stop point"),
// trained on the GPU with these hand-written kernels.
//
// Network (fixed shape): x[64] -> GELU(x W1 + b1)[256] -> GELU(h1 W2 + b2)[256]
// -> y = h2 W3 + b3, y estimating log2(stop nprobe).  Matrix products round both
// inputs to bf16 and accumulate in f32 (the bf16 arithmetic of the network);
// master weights, gradients and Adam moments are f32.
//
// Parameter vector layout (MLP_NPARAM floats): W1[64x256] b1[256] W2[256x256]
// b2[256] W3[256x1] b3[1]; row-major, y = x W + b.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/hy.h"
#include "hy_mlp.cuh"

namespace hy {
namespace {

__device__ inline float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// C[M x N] = op(A)[M x K] * op(B)[K x N] (+ C if accumulate), inputs rounded to
// bf16, f32 accumulation.  op(A)(m,k) = TA ? A[k*lda + m] : A[m*lda + k];
// op(B)(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n].  64 x 64 tile per CTA, 4 x 4
// outputs per thread, K in steps of 16.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_bf16_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                        const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                        int ldc, int accumulate) {
    __shared__ float As[16][68];
    __shared__ float Bs[16][68];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int i = threadIdx.x; i < 64 * 16; i += 256) {
            const int r = i >> 4, kk = i & 15;  // A tile: row r (m), column kk (k)
            const int m = m0 + r, k = k0 + kk;
            float a = 0.0f;
            if (m < M && k < K) a = TA ? A[static_cast<size_t>(k) * lda + m] : A[static_cast<size_t>(m) * lda + k];
            As[kk][r] = bf16r(a);
            const int n = n0 + r;  // B tile: column r (n), row kk (k)
            float b = 0.0f;
            if (n < N && k < K) b = TB ? B[static_cast<size_t>(n) * ldb + k] : B[static_cast<size_t>(k) * ldb + n];
            Bs[kk][r] = bf16r(b);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = As[kk][ty * 4 + u];
                b[u] = Bs[kk][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int m = m0 + ty * 4 + u;
        if (m >= M) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int n = n0 + tx * 4 + v;
            if (n >= N) continue;
            float* c = C + static_cast<size_t>(m) * ldc + n;
            *c = accumulate ? *c + acc[u][v] : acc[u][v];
        }
    }
}

__device__ inline float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ inline float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// Z += b (per column); A = GELU(Z) when act, else A = Z.
__global__ void bias_act_kernel(int M, int N, float* __restrict__ Z, const float* __restrict__ b,
                                float* __restrict__ A, int act) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<int64_t>(M) * N) return;
    const float z = Z[i] + b[i % N];
    Z[i] = z;
    A[i] = act ? gelu(z) : z;
}

// dZ = dA * GELU'(Z).
__global__ void act_grad_kernel(int64_t n, const float* __restrict__ Z, const float* __restrict__ dA,
                                float* __restrict__ dZ) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) dZ[i] = dA[i] * gelu_grad(Z[i]);
}

// db[n] = sum over rows of dZ[:, n].
__global__ void col_sum_kernel(int M, int N, const float* __restrict__ dZ, float* __restrict__ db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int m = 0; m < M; ++m) s += dZ[static_cast<size_t>(m) * N + n];
    db[n] = s;
}

// Mean squared error of y against t over M rows: loss (accumulated into
// *loss) and dy = 2 (y - t) / M.
__global__ void mse_kernel(int M, const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy,
                           float* __restrict__ loss) {
    __shared__ float red[256];
    float s = 0.0f;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        const float e = y[i] - t[i];
        dy[i] = 2.0f * e / static_cast<float>(M);
        s += e * e;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] / static_cast<float>(M);
}

__global__ void adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline int blocks(int64_t n, int t) { return static_cast<int>((n + t - 1) / t); }

template <bool TA, bool TB>
cudaError_t gemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc, int acc,
                 cudaStream_t s) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    gemm_bf16_kernel<TA, TB><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, acc);
    return cudaGetLastError();
}

}  // namespace

// Forward pass of B rows; keeps the pre-activations and activations for the
// backward pass.
cudaError_t mlp_forward(const float* params, int B, const float* X, MlpWork& w, float* y, cudaStream_t s) {
    const float* W1 = params + MLP_W1;
    const float* b1 = params + MLP_B1;
    const float* W2 = params + MLP_W2;
    const float* b2 = params + MLP_B2;
    const float* W3 = params + MLP_W3;
    const float* b3 = params + MLP_B3;
    cudaError_t e;
    if ((e = gemm<false, false>(B, MLP_H, MLP_IN, X, MLP_IN, W1, MLP_H, w.Z1, MLP_H, 0, s)) != cudaSuccess) return e;
    bias_act_kernel<<<blocks(static_cast<int64_t>(B) * MLP_H, 256), 256, 0, s>>>(B, MLP_H, w.Z1, b1, w.A1, 1);
    if ((e = gemm<false, false>(B, MLP_H, MLP_H, w.A1, MLP_H, W2, MLP_H, w.Z2, MLP_H, 0, s)) != cudaSuccess) return e;
    bias_act_kernel<<<blocks(static_cast<int64_t>(B) * MLP_H, 256), 256, 0, s>>>(B, MLP_H, w.Z2, b2, w.A2, 1);
    if ((e = gemm<false, false>(B, 1, MLP_H, w.A2, MLP_H, W3, 1, y, 1, 0, s)) != cudaSuccess) return e;
    bias_act_kernel<<<blocks(B, 256), 256, 0, s>>>(B, 1, y, b3, y, 0);
    return cudaGetLastError();
}

// Backward pass for dL/dy = dy (B values): gradients of every parameter into
// grads (overwritten).  Requires the activations of the matching forward.
cudaError_t mlp_backward(const float* params, int B, const float* X, MlpWork& w, const float* dy, float* grads,
                         cudaStream_t s) {
    const float* W2 = params + MLP_W2;
    const float* W3 = params + MLP_W3;
    cudaError_t e;
    // layer 3: dW3 = A2^T dy, db3 = sum dy, dA2 = dy W3^T
    if ((e = gemm<true, false>(MLP_H, 1, B, w.A2, MLP_H, dy, 1, grads + MLP_W3, 1, 0, s)) != cudaSuccess) return e;
    col_sum_kernel<<<1, 32, 0, s>>>(B, 1, dy, grads + MLP_B3);
    if ((e = gemm<false, true>(B, MLP_H, 1, dy, 1, W3, 1, w.dA, MLP_H, 0, s)) != cudaSuccess) return e;
    act_grad_kernel<<<blocks(static_cast<int64_t>(B) * MLP_H, 256), 256, 0, s>>>(static_cast<int64_t>(B) * MLP_H, w.Z2,
                                                                                 w.dA, w.dZ);
    // layer 2
    if ((e = gemm<true, false>(MLP_H, MLP_H, B, w.A1, MLP_H, w.dZ, MLP_H, grads + MLP_W2, MLP_H, 0, s)) != cudaSuccess)
        return e;
    col_sum_kernel<<<blocks(MLP_H, 128), 128, 0, s>>>(B, MLP_H, w.dZ, grads + MLP_B2);
    if ((e = gemm<false, true>(B, MLP_H, MLP_H, w.dZ, MLP_H, W2, MLP_H, w.dA, MLP_H, 0, s)) != cudaSuccess) return e;
    act_grad_kernel<<<blocks(static_cast<int64_t>(B) * MLP_H, 256), 256, 0, s>>>(static_cast<int64_t>(B) * MLP_H, w.Z1,
                                                                                 w.dA, w.dZ);
    // layer 1
    if ((e = gemm<true, false>(MLP_IN, MLP_H, B, X, MLP_IN, w.dZ, MLP_H, grads + MLP_W1, MLP_H, 0, s)) != cudaSuccess)
        return e;
    col_sum_kernel<<<blocks(MLP_H, 128), 128, 0, s>>>(B, MLP_H, w.dZ, grads + MLP_B1);
    return cudaGetLastError();
}

cudaError_t mlp_mse(int B, const float* y, const float* t, float* dy, float* loss, cudaStream_t s) {
    mse_kernel<<<1, 256, 0, s>>>(B, y, t, dy, loss);
    return cudaGetLastError();
}

cudaError_t mlp_adam(float* params, const float* grads, float* m, float* v, int step, float lr, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(step));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(step));
    adam_kernel<<<blocks(MLP_NPARAM, 256), 256, 0, s>>>(MLP_NPARAM, params, grads, m, v, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

size_t mlp_work_floats(int B) { return static_cast<size_t>(B) * MLP_H * 6; }

void mlp_work_bind(MlpWork& w, float* base, int B) {
    const size_t n = static_cast<size_t>(B) * MLP_H;
    w.Z1 = base;
    w.A1 = base + n;
    w.Z2 = base + 2 * n;
    w.A2 = base + 3 * n;
    w.dA = base + 4 * n;
    w.dZ = base + 5 * n;
}

}  // namespace hy

// Loss and gradients of the probe network on one batch (host pointers), for
// checking the training kernels.  No counterpart in the reference.
extern "C" int hy_mlp_loss_grad(const float* params, int B, const float* X, const float* t, float* loss,
                                float* grads) {
    if (!params || !X || !t || !loss || !grads || B < 1) return HY_ERR_ARG;
    float *dp = nullptr, *dX = nullptr, *dt = nullptr, *dy = nullptr, *ddy = nullptr, *dl = nullptr, *dg = nullptr,
          *dw = nullptr;
    int rc = HY_OK;
    auto al = [&](float** p, size_t n) {
        if (rc == HY_OK && cudaMalloc(p, n * sizeof(float)) != cudaSuccess) rc = HY_ERR_CUDA;
    };
    al(&dp, hy::MLP_NPARAM);
    al(&dX, static_cast<size_t>(B) * hy::MLP_IN);
    al(&dt, B);
    al(&dy, B);
    al(&ddy, B);
    al(&dl, 1);
    al(&dg, hy::MLP_NPARAM);
    al(&dw, hy::mlp_work_floats(B));
    if (rc == HY_OK) {
        cudaMemcpy(dp, params, hy::MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(dX, X, static_cast<size_t>(B) * hy::MLP_IN * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(dt, t, B * sizeof(float), cudaMemcpyHostToDevice);
        hy::MlpWork w;
        hy::mlp_work_bind(w, dw, B);
        cudaStream_t s = nullptr;
        if (hy::mlp_forward(dp, B, dX, w, dy, s) != cudaSuccess || hy::mlp_mse(B, dy, dt, ddy, dl, s) != cudaSuccess ||
            hy::mlp_backward(dp, B, dX, w, ddy, dg, s) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
            rc = HY_ERR_CUDA;
        if (rc == HY_OK) {
            cudaMemcpy(loss, dl, sizeof(float), cudaMemcpyDeviceToHost);
            cudaMemcpy(grads, dg, hy::MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost);
        }
    }
    for (float* p : {dp, dX, dt, dy, ddy, dl, dg, dw}) cudaFree(p);
    return rc;
}
