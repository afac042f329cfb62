// Diagnostic: one 128 x 128 x 128 bf16 tile through the tcgen05 path used by
// the batched scan (swizzled shared-memory operands, smem descriptors, MMA into
// TMEM, commit to an mbarrier, 32x32b loads), so the tests can check the
// tensor-core plumbing against an exact integer product on its own.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <string>

#include "../../include/hy.h"
#include "hy_tc.cuh"

namespace hy {
namespace {

// F8: operands are e4m3 (K = 256 in two 128-byte k-blocks), else bf16 (K = 128).
template <bool F8>
__global__ void __launch_bounds__(128) tc_selftest_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                                          float* __restrict__ D, int* err) {
    extern __shared__ unsigned char sm_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sA = base;          // 2 k-blocks x 16 KiB (128 rows)
    unsigned char* sB = base + 32768;  // 2 k-blocks x 16 KiB (128 columns of D)
    __shared__ uint64_t bar;
    __shared__ uint32_t tbase;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if constexpr (F8) {
        for (int i = threadIdx.x; i < 128 * 256; i += blockDim.x) {
            const int r = i >> 8, k = i & 255;
            const int kb = k >> 7, by = k & 127;
            const uint32_t off = kb * 16384 + r * 128 + ((((by >> 4) ^ (r & 7)) & 7) << 4) + (by & 15);
            sA[off] = __nv_cvt_float_to_fp8(A[i], __NV_SATFINITE, __NV_E4M3);
            sB[off] = __nv_cvt_float_to_fp8(B[i], __NV_SATFINITE, __NV_E4M3);
        }
    } else {
        for (int i = threadIdx.x; i < 128 * 128; i += blockDim.x) {
            const int r = i >> 7, k = i & 127;
            const int kb = k >> 6, kk = k & 63;
            *reinterpret_cast<__nv_bfloat16*>(sA + kb * 16384 + tc::kblock_offset(r, kk)) = __float2bfloat16_rn(A[i]);
            *reinterpret_cast<__nv_bfloat16*>(sB + kb * 16384 + tc::kblock_offset(r, kk)) = __float2bfloat16_rn(B[i]);
        }
    }
    fence_proxy_async();
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == 0) tc::tmem_alloc(&tbase, 128);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t t = tbase;
    if (threadIdx.x == 0) {
        const uint32_t idesc = F8 ? tc::idesc_e4m3_f32(128, 128) : tc::idesc_bf16_f32(128, 128);
        for (int kb = 0; kb < 2; ++kb)
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t a = tc::sdesc_sw128(smem_u32(sA + kb * 16384 + kk * 32));
                const uint64_t b = tc::sdesc_sw128(smem_u32(sB + kb * 16384 + kk * 32));
                if constexpr (F8)
                    tc::mma_e4m3(t, a, b, idesc, (kb | kk) != 0 ? 1u : 0u);
                else
                    tc::mma_bf16(t, a, b, idesc, (kb | kk) != 0 ? 1u : 0u);
            }
        tc::mma_commit(&bar);
    }
    __syncwarp();
    const bool ok = mbar_wait_bounded(&bar, 0, err);
    tc::fence_after_sync();
    if (ok) {
        for (int c = 0; c < 4; ++c) {
            float v[32];
            tc::tmem_ld32(t + (static_cast<uint32_t>(32 * warp) << 16) + c * 32, v);
            for (int j = 0; j < 32; ++j) D[(32 * warp + lane) * 128 + c * 32 + j] = v[j];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(t, 128);
}

}  // namespace
}  // namespace hy

namespace {

template <bool F8>
int run_selftest(const float* A, const float* B, float* D) {
    if (!A || !B || !D) return HY_ERR_ARG;
    float *dA = nullptr, *dB = nullptr, *dD = nullptr;
    int* derr = nullptr;
    const size_t in_bytes = (F8 ? 128 * 256 : 128 * 128) * sizeof(float);
    const size_t out_bytes = 128 * 128 * sizeof(float);
    int rc = HY_OK;
    if (cudaMalloc(&dA, in_bytes) != cudaSuccess || cudaMalloc(&dB, in_bytes) != cudaSuccess ||
        cudaMalloc(&dD, out_bytes) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
        rc = HY_ERR_CUDA;
    }
    if (rc == HY_OK) {
        cudaMemcpy(dA, A, in_bytes, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, B, in_bytes, cudaMemcpyHostToDevice);
        cudaMemset(dD, 0, out_bytes);
        cudaMemset(derr, 0, sizeof(int));
        const int smem = 65536 + 1024;
        cudaFuncSetAttribute(hy::tc_selftest_kernel<F8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        hy::tc_selftest_kernel<F8><<<1, 128, smem>>>(dA, dB, dD, derr);
        cudaError_t e = cudaDeviceSynchronize();
        int herr = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(D, dD, out_bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = HY_ERR_CUDA;
        else if (herr) rc = HY_ERR_TIMEOUT;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(derr);
    return rc;
}

}  // namespace

extern "C" int hy_selftest_tcgen05(const float* A, const float* B, float* D) { return run_selftest<false>(A, B, D); }

extern "C" int hy_selftest_tcgen05_e4m3(const float* A, const float* B, float* D) { return run_selftest<true>(A, B, D); }
