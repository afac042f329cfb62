// Device-side building blocks shared by the IVF kernels (sm_100a).
//
//  * ordered keys: a float score mapped to a uint32 whose unsigned order is the
//    float order; a 64-bit key (score << 32 | arena row) orders candidates by
//    score, then by arena row, so every selection here is deterministic;
//  * mbarrier + cp.async.bulk wrappers for staging list tiles in shared memory,
//    with bounded waits that report HY_ERR_TIMEOUT through a device flag
//    instead of spinning forever;
//  * warp-level bitonic sort / merge of KR*32 64-bit keys held in registers
//    (element e lives in lane e%32, register e/32), used as each warp's top-k.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hy {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint64_t KEY_MAX = ~0ull;
constexpr int TILE_ROWS = 32;        // rows per arena tile (one row per lane)
constexpr int PITCH_ALIGN = 32;      // dimension-block pitch granularity (floats)
constexpr int MAX_BLOCKS = 8;        // dimension blocks
constexpr uint32_t WAIT_LIMIT = 1u << 26;  // mbarrier polls before giving up

// Error codes written to the device status word (match HY_ERR_*).
constexpr int DEV_ERR_TIMEOUT = 4;
constexpr int DEV_ERR_ARG = 1;

__host__ __device__ inline uint32_t f2o(float f) {
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__host__ __device__ inline float o2f(uint32_t o) {
    uint32_t u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

__device__ inline uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ inline void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ inline void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ inline void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// 16-byte asynchronous copy global -> shared (L2 only), and the wait for
// every such copy this thread issued.  Both addresses 16-byte aligned.
__device__ inline void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// 4-byte asynchronous copy global -> shared (through L1), both addresses
// 4-byte aligned; cp_async_wait_all covers it too.
__device__ inline void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ inline void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Closes the group of this thread's asynchronous copies issued since the
// last commit (an empty group when there were none).
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most N of this thread's committed groups are still pending.
template <int N>
__device__ inline void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Plain arrival (count 1) on a CTA-local mbarrier.
__device__ inline void mbar_arrive_cta(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One 1-D bulk copy global -> shared, completing on `bar`.  dst, src 16-byte
// aligned; bytes a multiple of 16.
__device__ inline void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ inline bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`.  Returns false (and raises the
// device status word) if the phase did not complete within WAIT_LIMIT polls.
__device__ inline bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err) {
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicCAS(err, 0, DEV_ERR_TIMEOUT);
    return false;
}

__device__ inline uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__device__ inline uint64_t umax64(uint64_t a, uint64_t b) { return a < b ? b : a; }

// One compare-exchange layer of a bitonic network over KR*32 keys.
// `size` is the current bitonic block size (direction by (e & size)); pass
// size larger than every element index to sort everything ascending.
template <int KR>
__device__ inline void bitonic_layer(uint64_t (&v)[KR], int size, int stride, int lane) {
    if (stride >= 32) {
        const int rs = stride >> 5;
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            if ((r & rs) == 0) {
                const int e = r * 32 + lane;
                const bool up = (e & size) == 0;
                const uint64_t a = v[r], b = v[r | rs];
                const bool sw = up ? (a > b) : (a < b);
                v[r] = sw ? b : a;
                v[r | rs] = sw ? a : b;
            }
        }
    } else {
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const int e = r * 32 + lane;
            const bool up = (e & size) == 0;
            const uint64_t o = __shfl_xor_sync(FULL, v[r], stride);
            const bool lower = (lane & stride) == 0;
            v[r] = (lower == up) ? umin64(v[r], o) : umax64(v[r], o);
        }
    }
}

// Sort KR*32 keys ascending.
template <int KR>
__device__ inline void warp_sort(uint64_t (&v)[KR], int lane) {
#pragma unroll
    for (int size = 2; size <= KR * 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) bitonic_layer<KR>(v, size, stride, lane);
    }
}

// t (sorted ascending) := the KR*32 smallest of t U c, sorted ascending.
// c must be sorted ascending; it is consumed.
template <int KR>
__device__ inline void warp_merge(uint64_t (&t)[KR], uint64_t (&c)[KR], int lane) {
#pragma unroll
    for (int r = 0; r < KR; ++r) {
        const uint64_t rev = __shfl_sync(FULL, c[KR - 1 - r], 31 - lane);
        t[r] = umin64(t[r], rev);
    }
    // t is now bitonic; merge it ascending.
#pragma unroll
    for (int stride = KR * 16; stride > 0; stride >>= 1) bitonic_layer<KR>(t, KR * 64, stride, lane);
}

// Key at element index e (warp-uniform e), broadcast to every lane.
// (Each register is broadcast by its own shuffle and the wanted one kept: a
// select on e >> 5 would become an indexed access and put t in local memory.)
template <int KR>
__device__ inline uint64_t warp_get(const uint64_t (&t)[KR], int e) {
    uint64_t x = 0;
#pragma unroll
    for (int r = 0; r < KR; ++r) {
        const uint64_t v = __shfl_sync(FULL, t[r], e & 31);
        if (r == (e >> 5)) x = v;
    }
    return x;
}

}  // namespace hy
