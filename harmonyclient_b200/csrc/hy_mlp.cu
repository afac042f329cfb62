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
#include "hy_tc.cuh"

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

// ---------------------------------------------------------------------------
// Inference on the tensor cores.  The weights are packed once (mlp_pack) into
// the tcgen05 B-operand image: W1 as 256 rows (output features) x 64 inputs,
// one 128-byte-swizzled K-major k-block of 32 KiB; W2 as 256 rows x 256
// inputs, four such k-blocks.  One CTA of 1024 threads takes 128 queries
// (query = TMEM lane; eight threads per query split every layer's 256 columns):
// features -> bf16 A tile -> MMA (M 128, N 256,
// K 64) -> bias + GELU -> bf16 A tiles (4 k-blocks) -> MMA (K 256) -> bias +
// GELU -> dot with W3 -> nprobe, all on chip.
constexpr int MI_WIMG = 32768 + 4 * 32768;   // packed W1 + W2 bytes
constexpr int MI_SMEM = 1024 + 65536 + MI_WIMG;  // alignment slack, A tiles, weights

__global__ void mlp_pack_kernel(const float* __restrict__ params, unsigned char* __restrict__ wimg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_IN * MLP_H) {
        const int k = i / MLP_H, n = i % MLP_H;  // W1[k][n]
        *reinterpret_cast<__nv_bfloat16*>(wimg + tc::kblock_offset(n, k)) = __float2bfloat16_rn(params[MLP_W1 + i]);
    } else if (i < MLP_IN * MLP_H + MLP_H * MLP_H) {
        const int j = i - MLP_IN * MLP_H;
        const int k = j / MLP_H, n = j % MLP_H;  // W2[k][n]
        *reinterpret_cast<__nv_bfloat16*>(wimg + 32768 + (k >> 6) * 32768 + tc::kblock_offset(n, k & 63)) =
            __float2bfloat16_rn(params[MLP_W2 + j]);
    }
}

// 8 consecutive values as bf16 into one 16-byte chunk.
__device__ inline uint4 pack8_bf16(const float* v) {
    uint4 r;
    uint32_t* w = reinterpret_cast<uint32_t*>(&r);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 b = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        w[i] = *reinterpret_cast<const uint32_t*>(&b);
    }
    return r;
}

constexpr int MI_PARTS = 8;                 // threads per query row (column parts of every 256-wide layer)
constexpr int MI_COLS = MLP_H / MI_PARTS;   // columns of a layer per thread

__global__ void __launch_bounds__(128 * MI_PARTS, 1) mlp_infer_kernel(const float* __restrict__ pscore, int m, int P,
                                                           const float* __restrict__ mu, const float* __restrict__ sd,
                                                           const unsigned char* __restrict__ wimg,
                                                           const float* __restrict__ params, float margin,
                                                           int64_t* __restrict__ probes,
                                                           unsigned long long* __restrict__ total,
                                                           float* __restrict__ yout, int* err) {
    extern __shared__ unsigned char sm_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sA = base;             // 4 k-blocks x 128 rows x 128 B: X in k-block 0, then H1
    unsigned char* sW = base + 65536;     // W1 image (32 KiB) then W2 image (128 KiB)
    __shared__ uint64_t bar_w, bar_m;
    __shared__ uint32_t tbase;
    __shared__ int s_ok;
    // MI_PARTS threads per query row: warps w, w + 4, w + 8, ... share TMEM
    // lane quadrant w % 4 and take column parts 0, 1, ... (MI_COLS columns
    // each) of every 256-wide layer.
    const int warp = threadIdx.x >> 5, qt = warp >> 2;
    const int tid = threadIdx.x & 127;  // the query row within the tile
    const int row = blockIdx.x * 128 + tid;
    const bool valid = row < m;
    if (threadIdx.x == 0) {
        mbar_init(&bar_w, 1);
        mbar_init(&bar_m, 1);
        fence_mbar_init();
        s_ok = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar_w, MI_WIMG);
        for (int c = 0; c < MI_WIMG / 16384; ++c) bulk_g2s(sW + c * 16384, wimg + c * 16384, 16384, &bar_w);
    }
    if (warp == 0) tc::tmem_alloc(&tbase, 256);
    // Features of this thread's query (its P best coarse scores), standardised,
    // as bf16 row `tid` of the A tile.
    {
        const float* sc = pscore + static_cast<size_t>(valid ? row : 0) * P;
        const float s0 = valid ? sc[0] : 0.0f;
        const float a0 = fabsf(s0) + 1e-6f;
        constexpr int FC = 8 / MI_PARTS > 0 ? 8 / MI_PARTS : 1;  // 8-feature chunks per thread
#pragma unroll
        for (int c = FC * qt; c < FC * qt + FC; ++c) {
            float f[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int i = 8 * c + j;
                const float v = i == 0 ? logf(a0) : log1pf(fmaxf(sc[min(i, P - 1)] - s0, 0.0f) / a0);
                f[j] = valid ? (v - mu[i]) / sd[i] : 0.0f;
            }
            *reinterpret_cast<uint4*>(sA + tid * 128 + (((c ^ (tid & 7)) & 7) << 4)) = pack8_bf16(f);
        }
    }
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;
    const uint32_t idesc = tc::idesc_bf16_f32(128, 256);
    if (threadIdx.x == 0) {
        if (!mbar_wait_bounded(&bar_w, 0, err)) {
            s_ok = 0;
        } else {
            tc::fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                tc::mma_bf16(tmem, tc::sdesc_sw128(smem_u32(sA) + kk * 32), tc::sdesc_sw128(smem_u32(sW) + kk * 32),
                             idesc, kk != 0 ? 1u : 0u);
            tc::mma_commit(&bar_m);
        }
    }
    __syncthreads();
    bool ok = s_ok != 0 && mbar_wait_bounded(&bar_m, 0, err);
    tc::fence_after_sync();
    const uint32_t lane_addr = tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16);
    if (ok) {
        // Layer 1 epilogue: H1 = bf16(GELU(Z1 + b1)) into the 4 A k-blocks
        // (this thread's MI_COLS columns).
        {
            // 16 columns per TMEM load in a loop that is not unrolled: the
            // GELU code stays small enough for the instruction cache.
#pragma unroll 1
            for (int c2 = 0; c2 < MI_COLS / 16; ++c2) {
                const int col0 = MI_COLS * qt + 16 * c2;  // first of the 16 columns
                const int cb = col0 >> 6;                 // its A k-block
                uint32_t u[16];
                tc::tmem_ld16(lane_addr + col0, u);
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    const int c = ((col0 & 63) >> 3) + hh;  // 8-column chunk within the k-block
                    float h[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        h[j] = gelu(__uint_as_float(u[8 * hh + j]) + __ldg(params + MLP_B1 + col0 + 8 * hh + j));
                    *reinterpret_cast<uint4*>(sA + cb * 16384 + tid * 128 + (((c ^ (tid & 7)) & 7) << 4)) =
                        pack8_bf16(h);
                }
            }
        }
    }
    fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (threadIdx.x == 0 && ok) {
        for (int kb = 0; kb < 4; ++kb)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                tc::mma_bf16(tmem, tc::sdesc_sw128(smem_u32(sA + kb * 16384) + kk * 32),
                             tc::sdesc_sw128(smem_u32(sW + 32768 + kb * 32768) + kk * 32), idesc,
                             (kb | kk) != 0 ? 1u : 0u);
        tc::mma_commit(&bar_m);
    }
    __syncthreads();
    ok = ok && mbar_wait_bounded(&bar_m, 1, err);
    float acc = 0.0f;
    tc::fence_after_sync();
    if (ok) {
        // Layer 2 epilogue and layer 3: y = bf16(GELU(Z2 + b2)) . bf16(W3) + b3,
        // each thread over its MI_COLS columns.
        {
#pragma unroll 1
            for (int c2 = 0; c2 < MI_COLS / 16; ++c2) {
                const int col0 = MI_COLS * qt + 16 * c2;
                uint32_t u[16];
                tc::tmem_ld16(lane_addr + col0, u);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = col0 + j;
                    const float a = gelu(__uint_as_float(u[j]) + __ldg(params + MLP_B2 + n));
                    acc = fmaf(bf16r(a), bf16r(__ldg(params + MLP_W3 + n)), acc);
                }
            }
        }
        // Layer-3 partial sums of column parts 1.. in the A tiles' space: the
        // second MMA, which read them, has completed (bar_m).
        if (qt > 0) reinterpret_cast<float*>(sA)[(qt - 1) * 128 + tid] = acc;
    }
    __syncthreads();
    if (ok && qt == 0) {
        float y = acc;
#pragma unroll
        for (int j = 0; j < MI_PARTS - 1; ++j) y += reinterpret_cast<const float*>(sA)[j * 128 + tid];
        y += params[MLP_B3];
        if (valid) {
            if (yout) yout[row] = y;
            if (probes) {
                int np = static_cast<int>(ceilf(exp2f(fminf(y + margin, 30.0f))));
                np = max(1, min(P, np));
                for (int j = np; j < P; ++j) probes[static_cast<int64_t>(row) * P + j] = -1;
                atomicAdd(total, static_cast<unsigned long long>(np));
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 256);
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

size_t mlp_wimg_bytes() { return MI_WIMG; }

cudaError_t mlp_pack(const float* params, unsigned char* wimg, cudaStream_t s) {
    mlp_pack_kernel<<<blocks(MLP_IN * MLP_H + MLP_H * MLP_H, 256), 256, 0, s>>>(params, wimg);
    return cudaGetLastError();
}

cudaError_t mlp_infer(const float* pscore, int m, int P, const float* mu, const float* sd, const unsigned char* wimg,
                      const float* params, float margin, int64_t* probes, unsigned long long* total, float* yout,
                      int* err, cudaStream_t s) {
    if (m <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MI_SMEM);
    if (e != cudaSuccess) return e;
    mlp_infer_kernel<<<blocks(m, 128), 128 * MI_PARTS, MI_SMEM, s>>>(pscore, m, P, mu, sd, wimg, params, margin,
                                                                        probes, total, yout, err);
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
