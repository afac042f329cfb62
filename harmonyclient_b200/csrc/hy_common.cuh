// Device helpers shared by the scan kernels: exact sequential distance
// arithmetic, CTA-wide radix selection and bitonic sort in shared memory, query
// staging in the arena's block-padded layout and exact per-row distances read
// from the FP32 arena.
#pragma once
#include <cfloat>
#include <cstdint>

#include "hy_kernels.cuh"

namespace hy {

__device__ inline float sq_add(float acc, float a, float b) {
    const float t = __fsub_rn(a, b);
    return __fadd_rn(acc, __fmul_rn(t, t));
}
__device__ inline float ip_add(float acc, float a, float b) { return __fadd_rn(acc, __fmul_rn(a, b)); }


// ---------------------------------------------------------------------------
// CTA-wide radix selection over n ordered uint32 values in shared memory:
// returns v*, the m-th smallest value (1 <= m <= n), and through *need the
// number of elements equal to v* that belong to the m smallest.
__device__ inline uint32_t cta_radix_select(const uint32_t* vals, int n, int m, int* need, int* hist /*256*/,
                                     uint32_t* sh /*2*/) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        sh[0] = 0;                        // prefix
        sh[1] = static_cast<uint32_t>(m);  // remaining
    }
    __syncthreads();
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 24 - 8 * pass;
        for (int i = tid; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const uint32_t prefix = sh[0];
        for (int i = tid; i < n; i += blockDim.x) {
            const uint32_t v = vals[i];
            if (pass == 0 || (v >> (shift + 8)) == (prefix >> (shift + 8))) atomicAdd(&hist[(v >> shift) & 255], 1);
        }
        __syncthreads();
        if (tid < 32) {
            const int lane = tid;
            int loc[8];
            int sum = 0;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                loc[u] = hist[lane * 8 + u];
                sum += loc[u];
            }
            int incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += t;
            }
            const int excl = incl - sum;
            const int rem = static_cast<int>(sh[1]);
            const bool mine = excl < rem && incl >= rem;
            const unsigned who = __ballot_sync(FULL, mine);
            if (mine) {
                int cum = excl;
                int digit = lane * 8 + 7;
                int before = excl;
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (cum + loc[u] >= rem) {
                        digit = lane * 8 + u;
                        before = cum;
                        break;
                    }
                    cum += loc[u];
                }
                sh[0] = prefix | (static_cast<uint32_t>(digit) << shift);
                sh[1] = static_cast<uint32_t>(rem - before);
            }
            (void)who;
        }
        __syncthreads();
    }
    const uint32_t v = sh[0];
    *need = static_cast<int>(sh[1]);
    __syncthreads();
    return v;
}

// Collect the m smallest (value, index) pairs of vals[0..n) as 64-bit keys
// (value << 32 | index) into sel[0..m): everything below v*, then the `need`
// lowest-index elements equal to v*.  Order inside sel is unspecified.
__device__ inline void cta_collect(const uint32_t* vals, int n, int m, uint32_t vstar, int need, uint64_t* sel,
                            int* scratch /*34*/) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    int* cnt_lt = scratch;      // [0]
    int* taken = scratch + 1;   // [1]
    int* wcnt = scratch + 2;    // [2..33]
    if (tid == 0) {
        *cnt_lt = 0;
        *taken = 0;
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
        const uint32_t v = vals[i];
        if (v < vstar) {
            const int pos = atomicAdd(cnt_lt, 1);
            sel[pos] = (static_cast<uint64_t>(v) << 32) | static_cast<uint32_t>(i);
        }
    }
    const int base_eq = m - need;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + tid;
        const bool f = i < n && vals[i] == vstar;
        const unsigned b = __ballot_sync(FULL, f);
        if (lane == 0) wcnt[warp] = __popc(b);
        __syncthreads();
        int pre = 0, tot = 0;
        for (int w = 0; w < nw; ++w) {
            const int c = wcnt[w];
            if (w < warp) pre += c;
            tot += c;
        }
        const int r = *taken + pre + __popc(b & ((1u << lane) - 1u));
        if (f && r < need) sel[base_eq + r] = (static_cast<uint64_t>(vstar) << 32) | static_cast<uint32_t>(i);
        __syncthreads();
        if (tid == 0) *taken += tot;
        __syncthreads();
        if (*taken >= need) break;
    }
    __syncthreads();
}

// In-place ascending bitonic sort of P (power of two) keys in shared memory.
__device__ inline void cta_bitonic_sort(uint64_t* a, int P) {
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < P / 2; i += blockDim.x) {
                const int lo = 2 * i - (i & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint64_t x = a[lo], y = a[hi];
                if ((x > y) == up) {
                    a[lo] = y;
                    a[hi] = x;
                }
            }
            __syncthreads();
        }
    }
}

// k-th smallest of the warp's values v (lane l holds elements r*32 + l, valid
// below n): four 8-bit radix passes over a per-warp 256-bin histogram.
template <int PER>
__device__ inline uint32_t warp_radix_select(const uint32_t (&v)[PER], int n, int k, int* hist, int lane) {
    uint32_t prefix = 0, mask = 0;
    int rem = k;
#pragma unroll 1
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 24 - 8 * pass;
#pragma unroll
        for (int i = 0; i < 8; ++i) hist[lane * 8 + i] = 0;
        __syncwarp();
#pragma unroll
        for (int r = 0; r < PER; ++r)
            if (r * 32 + lane < n && (v[r] & mask) == prefix) atomicAdd(&hist[(v[r] >> shift) & 255u], 1);
        __syncwarp();
        int loc[8], sum = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            loc[i] = hist[lane * 8 + i];
            sum += loc[i];
        }
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        const int excl = incl - sum;
        const bool mine = excl < rem && incl >= rem;
        int digit = 0, before = 0;
        if (mine) {
            int cum = excl;
            digit = lane * 8 + 7;
            before = excl;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (cum + loc[i] >= rem) {
                    digit = lane * 8 + i;
                    before = cum;
                    break;
                }
                cum += loc[i];
            }
        }
        const unsigned who = __ballot_sync(FULL, mine);
        const int src = __ffs(who) - 1;
        digit = __shfl_sync(FULL, digit, src);
        before = __shfl_sync(FULL, before, src);
        prefix |= static_cast<uint32_t>(digit) << shift;
        mask |= 0xffu << shift;
        rem -= before;
        __syncwarp();
    }
    return prefix;
}

// An upper bound U on the k-th smallest of the warp's values (k <= n; lane l
// holds elements r*32 + l, valid below n) with at least k values <= U: two
// 8-bit radix passes over the bits below the prefix that every value shares
// (found from the warp's minimum and maximum), so the passes split the values'
// actual range; U is the upper edge of the bin that holds the k-th value,
// within 2^(top - 15) of it in the ordered-bits order (top = the highest bit
// in which the values differ).
template <int PER>
__device__ inline uint32_t warp_select_bound(const uint32_t (&v)[PER], int n, int k, int* hist, int lane) {
    uint32_t mn = 0xffffffffu, mx = 0u;
#pragma unroll
    for (int r = 0; r < PER; ++r)
        if (r * 32 + lane < n) {
            mn = min(mn, v[r]);
            mx = max(mx, v[r]);
        }
    mn = __reduce_min_sync(FULL, mn);
    mx = __reduce_max_sync(FULL, mx);
    if (mn == mx) return mn;
    int top = 31 - __clz(mn ^ mx);  // highest differing bit
    uint32_t mask = ~((2u << top) - 1u);
    uint32_t prefix = mn & mask;
    int rem = k;
#pragma unroll 1
    for (int pass = 0; pass < 2 && top >= 0; ++pass) {
        const int shift = top > 7 ? top - 7 : 0;
        const uint32_t wmask = ((2u << top) - 1u) & ~((1u << shift) - 1u);  // bits [shift, top]
#pragma unroll
        for (int i = 0; i < 8; ++i) hist[lane * 8 + i] = 0;
        __syncwarp();
#pragma unroll
        for (int r = 0; r < PER; ++r)
            if (r * 32 + lane < n && (v[r] & mask) == prefix) atomicAdd(&hist[(v[r] & wmask) >> shift], 1);
        __syncwarp();
        int loc[8], sum = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            loc[i] = hist[lane * 8 + i];
            sum += loc[i];
        }
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        const int excl = incl - sum;
        const bool mine = excl < rem && incl >= rem;
        int digit = 0, before = 0;
        if (mine) {
            int cum = excl;
            digit = lane * 8 + 7;
            before = excl;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (cum + loc[i] >= rem) {
                    digit = lane * 8 + i;
                    before = cum;
                    break;
                }
                cum += loc[i];
            }
        }
        const unsigned who = __ballot_sync(FULL, mine);
        const int src = __ffs(who) - 1;
        digit = __shfl_sync(FULL, digit, src);
        before = __shfl_sync(FULL, before, src);
        prefix |= static_cast<uint32_t>(digit) << shift;
        mask |= wmask;
        rem -= before;
        top = shift - 1;
        __syncwarp();
    }
    return top >= 0 ? (prefix | ((2u << top) - 1u)) : prefix;
}

__host__ __device__ inline int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// ---------------------------------------------------------------------------
// Copy query `qi` into shared memory in the arena's block-padded layout
// (block b at boff[b], zero padding up to its pitch).
__device__ inline void stage_query(const ArenaLayout& L, const float* __restrict__ q, float* qs) {
    for (int i = threadIdx.x; i < L.row_pitch; i += blockDim.x) {
        int b = 0;
        while (b + 1 < L.nb && i >= L.boff[b + 1]) ++b;
        const int j = i - L.boff[b];
        const int w = L.bstart[b + 1] - L.bstart[b];
        qs[i] = j < w ? q[L.bstart[b] + j] : 0.0f;
    }
}

// Squared L2 of one arena row against the staged query, read straight from
// global memory; blockwise = sum each dimension block from zero and add the
// block sums (the scan's order), else one running sum over all dimensions
// (the reference's lite_scan_codes order, src/utils.h:480-487).
__device__ inline float row_l2_global(const ArenaLayout& L, const float* __restrict__ codes, int64_t r,
                                      const float* qs, bool blockwise) {
    float total = 0.0f;
    const int lr = static_cast<int>(r & 31);
    const float* tile = codes + static_cast<size_t>(r >> 5) * 32 * L.row_pitch;
    for (int b = 0; b < L.nb; ++b) {
        const float* rowp = tile + static_cast<size_t>(L.boff[b]) * 32 + static_cast<size_t>(lr) * L.pitch[b];
        const float* qb = qs + L.boff[b];
        const int w = L.bstart[b + 1] - L.bstart[b];
        float s = blockwise ? 0.0f : total;
        for (int c = 0; c * 4 < w; ++c) {
            const int pc = (c & ~7) | ((c ^ lr) & 7);
            const float4 x = __ldg(reinterpret_cast<const float4*>(rowp + pc * 4));
            const float4 y = *reinterpret_cast<const float4*>(qb + c * 4);
            const int j = c * 4;
            s = sq_add(s, y.x, x.x);
            if (j + 1 < w) s = sq_add(s, y.y, x.y);
            if (j + 2 < w) s = sq_add(s, y.z, x.z);
            if (j + 3 < w) s = sq_add(s, y.w, x.w);
        }
        total = blockwise ? (b == 0 ? s : __fadd_rn(total, s)) : s;
    }
    return total;
}


// Inner product of one arena row with the staged query, sequential float sum
// over the blocks in order (the plain scan's IP arithmetic).
__device__ inline float row_ip_global(const ArenaLayout& L, const float* __restrict__ codes, int64_t r,
                                      const float* qs) {
    float total = 0.0f;
    const int lr = static_cast<int>(r & 31);
    const float* tile = codes + static_cast<size_t>(r >> 5) * 32 * L.row_pitch;
    for (int b = 0; b < L.nb; ++b) {
        const float* rowp = tile + static_cast<size_t>(L.boff[b]) * 32 + static_cast<size_t>(lr) * L.pitch[b];
        const float* qb = qs + L.boff[b];
        const int w = L.bstart[b + 1] - L.bstart[b];
        float s = 0.0f;
        for (int j = 0; j < w; ++j) {
            const int c = j >> 2;
            const int pc = (c & ~7) | ((c ^ lr) & 7);
            s = __fadd_rn(s, __fmul_rn(qb[j], __ldg(rowp + pc * 4 + (j & 3))));
        }
        total = b == 0 ? s : __fadd_rn(total, s);
    }
    return total;
}

}  // namespace hy
