// Batched list-major scan on the tcgen05 tensor cores (the "bf16" and
// "e4m3" forms) and the steps around it.
//
// Queries that probe the same list share one pass over it.  After coarse
// quantisation, the (query, probed list) pairs are inverted into per-list
// query groups; a persistent kernel (one CTA per SM) drains a work queue of
// (list, group of <=128 queries, slice of <=2048 rows) items.  Per item the
// CTA gathers the group's query vectors into shared memory (the MMA's B
// operand), then streams the slice's 128-row tiles of the list image (already
// in the tensor core's swizzled shared-memory layout, so each k-block of a
// tile is one 16 KiB bulk copy) through a ring of stages.  One thread issues
// tcgen05.mma (M = 128 rows, N = up to 128 queries) into one of two TMEM
// accumulators; eight epilogue warps read the accumulator (thread = row) and
// form dist = |x|^2 + |q|^2 - 2 q.x (or -q.x for inner product) with a
// rigorous bound on its distance from the plain scan's exact FP32 value.
//
// First pass (each query's nearest list): dense items write the distance of
// every row; the tightening step recomputes each row's bound, takes each
// query's k-th smallest dist + bound as its threshold and keeps the rows
// whose dist - bound reach it.  Second pass (the other probed lists): rows whose dist - bound passes
// the threshold are emitted as candidates.  The re-rank keeps the candidates
// whose bound can reach the top-k and gives them the exact FP32 distance (or
// keeps the tensor-core distance when the exactness certificate shows it is
// exact), so the answer is the plain scan's.  A query whose candidates
// overflow its buffer is answered again by the plain scan.  The same kernel,
// over the centroids as a one-list index, is the coarse step of the bf16 form.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cfloat>
#include <cstddef>

#include "hy_batched.cuh"
#include "hy_common.cuh"
#include "hy_tc.cuh"

namespace hy {
namespace {

constexpr int METRIC_IP = 0, METRIC_L2 = 1;  // include/hy.h's HY_METRIC_*
constexpr int TM = 128;      // rows per tile (MMA M)
constexpr int NS_MIN = 4;    // A stages (one 16 KiB k-block each): at least this many,
constexpr int NS_MAX = 8;    // and as many more as shared memory holds
constexpr int KB_BYTES = 16384;

// ---------------------------------------------------------------------------
// Conversion of the FP32 arena into the bf16 tensor-core image.
__global__ void to_bf16_arena_kernel(ArenaLayout L, const float* __restrict__ codes, int64_t rows, int nkb,
                                     unsigned char* __restrict__ out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= rows * L.d) return;
    const int64_t r = i / L.d;
    const int j = static_cast<int>(i % L.d);
    int b = 0;
    while (b + 1 < L.nb && j >= L.bstart[b + 1]) ++b;
    const float v = codes[arena_offset(L, r, b, j - L.bstart[b])];
    const int64_t tile = r >> 7;
    const int kb = j >> 6;
    unsigned char* dst = out + (tile * nkb + kb) * KB_BYTES + tc::kblock_offset(static_cast<uint32_t>(r & 127), j & 63);
    *reinterpret_cast<__nv_bfloat16*>(dst) = __float2bfloat16_rn(v);
}

// e4m3 code of v / scale and its decoded value times scale (saturating at
// the largest finite e4m3 magnitude, 448).
__device__ inline unsigned char e4m3_code(float v, float scale) {
    return static_cast<unsigned char>(__nv_cvt_float_to_fp8(v / scale, __NV_SATFINITE, __NV_E4M3));
}
__device__ inline float e4m3_value(unsigned char c, float scale) {
    const __half_raw h = __nv_cvt_fp8_to_halfraw(static_cast<__nv_fp8_storage_t>(c), __NV_E4M3);
    return __half2float(__half(h)) * scale;
}

// e4m3 image of the arena: per 128-row tile, ceil(d/128) k-blocks of 128 rows
// x 128 bytes in the same swizzled K-major layout as the bf16 image; every
// value is coded relative to its list's scale (tscale of its tile).
__global__ void to_f8_arena_kernel(ArenaLayout L, const float* __restrict__ codes, int64_t rows, int nkb,
                                   const float* __restrict__ tscale, unsigned char* __restrict__ out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= rows * L.d) return;
    const int64_t r = i / L.d;
    const int j = static_cast<int>(i % L.d);
    int b = 0;
    while (b + 1 < L.nb && j >= L.bstart[b + 1]) ++b;
    const float v = codes[arena_offset(L, r, b, j - L.bstart[b])];
    const int64_t tile = r >> 7;
    const uint32_t row = static_cast<uint32_t>(r & 127), by = static_cast<uint32_t>(j & 127);
    out[(tile * nkb + (j >> 7)) * KB_BYTES + row * 128u + ((((by >> 4) ^ (row & 7u)) & 7u) << 4) + (by & 15u)] =
        e4m3_code(v, tscale[tile]);
}

// Largest |value| of each 128-row tile (one warp per tile).
__global__ void tile_absmax_kernel(ArenaLayout L, const float* __restrict__ codes, int64_t tiles,
                                   float* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t t = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (t >= tiles) return;
    float m = 0.0f;
    for (int r = 0; r < TM; ++r)
        for (int j = lane; j < L.d; j += 32) {
            int b = 0;
            while (b + 1 < L.nb && j >= L.bstart[b + 1]) ++b;
            m = fmaxf(m, fabsf(codes[arena_offset(L, t * TM + r, b, j - L.bstart[b])]));
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if (lane == 0) out[t] = m;
}

// Per list: scale = (largest |value| over its tiles) / 448, 1 for an all-zero
// list; the list's tiles get the same scale.
__global__ void list_scale_kernel(const int64_t* __restrict__ list_off, const int32_t* __restrict__ list_size,
                                  int nlist, const float* __restrict__ tile_max, float* __restrict__ lscale,
                                  float* __restrict__ tscale) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlist) return;
    const int64_t t0 = list_off[l] / TM;
    const int nt = (list_size[l] + TM - 1) / TM;
    float m = 0.0f;
    for (int t = 0; t < nt; ++t) m = fmaxf(m, tile_max[t0 + t]);
    const float sc = m > 0.0f ? m / 448.0f : 1.0f;
    lscale[l] = sc;
    for (int t = 0; t < nt; ++t) tscale[t0 + t] = sc;
}

// Per-row quantities for the error bound: |x~| (norm of the row as the tensor
// cores see it: bf16-rounded, or e4m3-coded times its tile's scale when
// tscale is given) and |x - x~| (its rounding error), one warp per arena row.
__global__ void row_aux_kernel(ArenaLayout L, const float* __restrict__ codes, int64_t rows,
                               const float* __restrict__ tscale, float2* __restrict__ aux) {
    const int lane = threadIdx.x & 31;
    const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (r >= rows) return;
    float nn = 0.0f, ee = 0.0f;
    const float ts = tscale ? tscale[r >> 7] : 1.0f;
    for (int j = lane; j < L.d; j += 32) {
        int b = 0;
        while (b + 1 < L.nb && j >= L.bstart[b + 1]) ++b;
        const float v = codes[arena_offset(L, r, b, j - L.bstart[b])];
        const float vb = tscale ? e4m3_value(e4m3_code(v, ts), ts) : __bfloat162float(__float2bfloat16_rn(v));
        nn = fmaf(vb, vb, nn);
        ee = fmaf(v - vb, v - vb, ee);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nn += __shfl_xor_sync(FULL, nn, o);
        ee += __shfl_xor_sync(FULL, ee, o);
    }
    if (lane == 0) aux[r] = make_float2(sqrtf(nn), sqrtf(ee));
}

// Per 128-row tile: the largest |x~| and |x - x~| of its rows (the batched
// kernel's per-tile relaxation of the error bound).
__global__ void tile_aux_kernel(const float2* __restrict__ row_aux, int64_t tiles, float2* __restrict__ out) {
    const int64_t t = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= tiles) return;
    float a = 0.0f, e = 0.0f;
    for (int r = lane; r < TM; r += 32) {
        const float2 v = row_aux[t * TM + r];
        a = fmaxf(a, v.x);
        e = fmaxf(e, v.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fmaxf(a, __shfl_xor_sync(FULL, a, o));
        e = fmaxf(e, __shfl_xor_sync(FULL, e, o));
    }
    if (lane == 0) out[t] = make_float2(a, e);
}

// Per 128-row tile: the largest squared norm of its rows.
__global__ void tile_max_kernel(const float* __restrict__ xn, int64_t tiles, float* __restrict__ out) {
    const int64_t t = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= tiles) return;
    float m = 0.0f;
    for (int r = lane; r < TM; r += 32) m = fmaxf(m, xn[t * TM + r]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if (lane == 0) out[t] = m;
}

// Queries in e4m3: per query scale t = max|q_j| / 448 (1 for a zero query),
// codes of q_j / t padded to nkb*128 bytes, and {|q|^2, |q|, |q~|, |q - q~|}
// with q~ = t * decoded code.
__global__ void prep_queries_f8_kernel(const float* __restrict__ q, int nq, int d, int nkb,
                                       unsigned char* __restrict__ qb, float4* __restrict__ qaux,
                                       float* __restrict__ qscale) {
    const int i = blockIdx.x;
    if (i >= nq) return;
    const float* src = q + static_cast<size_t>(i) * d;
    __shared__ float red[2][4];
    __shared__ float s_t;
    float m = 0.0f;
    for (int j = threadIdx.x; j < d; j += blockDim.x) m = fmaxf(m, fabsf(src[j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0) red[0][threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mm = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mm = fmaxf(mm, red[0][w]);
        s_t = mm > 0.0f ? mm / 448.0f : 1.0f;
    }
    __syncthreads();
    const float t = s_t;
    float nn = 0.0f, ee = 0.0f;
    for (int j = threadIdx.x; j < nkb * 128; j += blockDim.x) {
        const float v = j < d ? src[j] : 0.0f;
        const unsigned char c = e4m3_code(v, t);
        qb[static_cast<size_t>(i) * nkb * 128 + j] = c;
        const float vb = e4m3_value(c, t);
        nn = fmaf(vb, vb, nn);
        ee = fmaf(v - vb, v - vb, ee);
    }
    __syncthreads();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nn += __shfl_xor_sync(FULL, nn, o);
        ee += __shfl_xor_sync(FULL, ee, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = nn;
        red[1][threadIdx.x >> 5] = ee;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int j = 0; j < d; ++j) s = __fadd_rn(s, __fmul_rn(src[j], src[j]));
        float tn = 0.0f, te = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            tn += red[0][w];
            te += red[1][w];
        }
        qaux[i] = make_float4(s, sqrtf(s), sqrtf(tn), sqrtf(te));
        qscale[i] = t;
    }
}

// Queries: bf16 rows padded to nkb*64, and per query {|q|^2 (sequential f32,
// the exact arithmetic's value), |q|, |q~|, |q - q~|}.  One warp per query
// (PREP_WARPS per CTA): the lanes convert and reduce, and lane 0 takes the
// sequential sum from the row staged in shared memory.
constexpr int PREP_WARPS = 8;
constexpr int PREP_DMAX = 768;  // the bf16 forms' largest d
__global__ void __launch_bounds__(32 * PREP_WARPS) prep_queries_kernel(const float* __restrict__ q, int nq, int d,
                                                                       int nkb, __nv_bfloat16* __restrict__ qb,
                                                                       float4* __restrict__ qaux, float amax,
                                                                       int32_t* __restrict__ qexact) {
    __shared__ float rowbuf[PREP_WARPS][PREP_DMAX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * PREP_WARPS + warp;
    if (i >= nq) return;  // whole warp
    const float* src = q + static_cast<size_t>(i) * d;
    float* row = rowbuf[warp];
    float nn = 0.0f, ee = 0.0f;
    bool integral = true;
    for (int j = lane; j < nkb * 64; j += 32) {
        const float v = j < d ? src[j] : 0.0f;
        if (j < d) row[j] = v;
        integral = integral && v == rintf(v) && fabsf(v) <= 256.0f;
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        qb[static_cast<size_t>(i) * nkb * 64 + j] = b;
        const float vb = __bfloat162float(b);
        nn = fmaf(vb, vb, nn);
        ee = fmaf(v - vb, v - vb, ee);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nn += __shfl_xor_sync(FULL, nn, o);
        ee += __shfl_xor_sync(FULL, ee, o);
    }
    const bool all_integral = __all_sync(FULL, integral);
    __syncwarp();
    if (lane == 0) {
        float s = 0.0f;
#pragma unroll 8
        for (int j = 0; j < d; ++j) s = __fadd_rn(s, __fmul_rn(row[j], row[j]));
        qaux[i] = make_float4(s, sqrtf(s), sqrtf(nn), sqrtf(ee));
        if (qexact) qexact[i] = (amax >= 0.0f && all_integral && s + amax < 8388608.0f) ? 1 : 0;
    }
}

// Exactness certificate of the bf16 image: flag = every arena value is an
// integer of magnitude at most 256 (exact in bf16); maxxn = the largest row
// squared norm (bit pattern of a non-negative float).
__global__ void arena_integral_kernel(const float* __restrict__ codes, int64_t n, const float* __restrict__ xn,
                                      int64_t rows, int* __restrict__ flag, unsigned int* __restrict__ maxxn) {
    bool ok = true;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float v = codes[i];
        ok = ok && v == rintf(v) && fabsf(v) <= 256.0f;
    }
    unsigned int mx = 0u;
    for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < rows;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x)
        mx = max(mx, __float_as_uint(xn[r]));
    if (!__syncthreads_and(ok ? 1 : 0) && threadIdx.x == 0) atomicAnd(flag, 0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(FULL, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxxn, mx);
}

// Bound on |bf16 distance - exact FP32 distance| for one (query, row) pair,
// the exact distance being the plain scan's sequential f32 sum.  With x~, q~
// the bf16-rounded vectors: |x~.q~ - x.q| <= |x~||q - q~| + |q||x - x~|; the
// f32 accumulation of K products adds at most cK |x~||q~| (cK = (K+8) 2^-24);
// the f32 norms, the final |x|^2 + |q|^2 - 2 x.q and the plain scan's own
// d-term sum add at most cN (|x|^2 + |q|^2) (cN = (3d+16) 2^-24).  L2 doubles
// the inner-product terms.  Both constants carry a 2^-7 inflation for the
// rounding of the bound itself (set on the host).
struct ErrCoef {
    float aq, bq, cq;  // per query: multiplies |x~|, multiplies |x - x~|, constant
};
__device__ inline ErrCoef err_coef(float4 qa, bool l2, float cK, float cN) {
    const float inflate = 1.0f + 0.0078125f;
    ErrCoef c;
    if (l2) {
        c.aq = inflate * 2.0f * (qa.w + cK * qa.z);
        c.bq = inflate * 2.0f * qa.y;
        c.cq = cN * qa.x;
    } else {
        c.aq = inflate * (qa.w + (cK + cN) * qa.z);
        c.bq = inflate * qa.y;
        c.cq = 0.0f;
    }
    return c;
}
__device__ inline float err_row_const(float xn, bool l2, float cN) { return l2 ? cN * xn : 0.0f; }

// ---------------------------------------------------------------------------
// Inverting the probe lists.
// Only probe columns [j0, j1) of each query take part (probe rank ranges).
__global__ void probe_hist_kernel(const int64_t* __restrict__ probes, int nq, int nprobe, int j0, int j1,
                                  int32_t* __restrict__ cnt) {
    const int w = j1 - j0;
    const int64_t n = static_cast<int64_t>(nq) * w;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t l = probes[(i / w) * nprobe + j0 + i % w];
        if (l >= 0) atomicAdd(&cnt[l], 1);
    }
}

// Single-CTA exclusive scan of n int32 counts into int64 offsets (n+1 entries).
__global__ void __launch_bounds__(1024) scan_kernel(const int32_t* __restrict__ in, int n, int64_t* __restrict__ out) {
    __shared__ int64_t part[1024];
    const int t = threadIdx.x;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int a = min(n, t * per), b = min(n, a + per);
    int64_t s = 0;
    for (int i = a; i < b; ++i) s += in[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
        const int64_t v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int64_t run = part[t] - s;
    for (int i = a; i < b; ++i) {
        out[i] = run;
        run += in[i];
    }
    if (t == blockDim.x - 1) out[n] = part[t];
}

__global__ void probe_fill_kernel(const int64_t* __restrict__ probes, int nq, int nprobe, int j0, int j1,
                                  const int64_t* __restrict__ off, int32_t* __restrict__ fill,
                                  int32_t* __restrict__ pairs) {
    const int w = j1 - j0;
    const int64_t n = static_cast<int64_t>(nq) * w;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t l = probes[(i / w) * nprobe + j0 + i % w];
        if (l < 0) continue;
        const int pos = atomicAdd(&fill[l], 1);
        pairs[off[l] + pos] = static_cast<int32_t>(i / w);
    }
}

// The same two steps with shared-memory counters (nlist <= INVERT_SMEM_LISTS):
// each CTA takes a contiguous range of `per` pairs, counts them per list in
// shared memory and adds each list's count to the global one once; the fill
// reserves each list's share of the CTA with one global add and places the
// pairs at shared-memory ranks.  Few global atomics per list instead of one
// per pair.
constexpr int INVERT_SMEM_LISTS = 6144;  // the fill's 8 bytes per list stay within 48 KiB
__global__ void __launch_bounds__(512) probe_hist_smem_kernel(const int64_t* __restrict__ probes, int nq, int nprobe,
                                                              int j0, int j1, int nlist, int64_t per,
                                                              int32_t* __restrict__ cnt) {
    extern __shared__ int h[];  // [nlist]
    const int w = j1 - j0;
    const int64_t n = static_cast<int64_t>(nq) * w;
    const int64_t a = blockIdx.x * per, b = min(n, a + per);
    for (int l = threadIdx.x; l < nlist; l += blockDim.x) h[l] = 0;
    __syncthreads();
    for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) {
        const int64_t l = probes[(i / w) * nprobe + j0 + i % w];
        if (l >= 0) atomicAdd(&h[l], 1);
    }
    __syncthreads();
    for (int l = threadIdx.x; l < nlist; l += blockDim.x)
        if (h[l]) atomicAdd(&cnt[l], h[l]);
}

__global__ void __launch_bounds__(512) probe_fill_smem_kernel(const int64_t* __restrict__ probes, int nq, int nprobe,
                                                              int j0, int j1, int nlist, int64_t per,
                                                              const int64_t* __restrict__ off,
                                                              int32_t* __restrict__ fill,
                                                              int32_t* __restrict__ pairs) {
    extern __shared__ int h[];  // [nlist] counts, then ranks; [nlist] bases
    int* base = h + nlist;
    const int w = j1 - j0;
    const int64_t n = static_cast<int64_t>(nq) * w;
    const int64_t a = blockIdx.x * per, b = min(n, a + per);
    for (int l = threadIdx.x; l < nlist; l += blockDim.x) h[l] = 0;
    __syncthreads();
    for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) {
        const int64_t l = probes[(i / w) * nprobe + j0 + i % w];
        if (l >= 0) atomicAdd(&h[l], 1);
    }
    __syncthreads();
    for (int l = threadIdx.x; l < nlist; l += blockDim.x) {
        base[l] = h[l] ? atomicAdd(&fill[l], h[l]) : 0;
        h[l] = 0;
    }
    __syncthreads();
    for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) {
        const int64_t l = probes[(i / w) * nprobe + j0 + i % w];
        if (l < 0) continue;
        const int pos = base[l] + atomicAdd(&h[l], 1);
        pairs[off[l] + pos] = static_cast<int32_t>(i / w);
    }
}

// Items of a list = query groups x row slices (none for an empty list).
__global__ void item_count_kernel(const int32_t* __restrict__ cnt, const int32_t* __restrict__ list_size, int nlist,
                                  int rs, int qg, int32_t* __restrict__ items) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlist) return;
    const int c = cnt[l], s = list_size[l];
    items[l] = (c > 0 && s > 0) ? ((c + qg - 1) / qg) * ((s + rs - 1) / rs) : 0;
}

// Item descriptors {list, query group, row slice} for the first `cap` items,
// so the batched kernel decodes an item with one load (one warp per list).
__global__ void item_fill_kernel(const int64_t* __restrict__ item_off, const int32_t* __restrict__ list_size,
                                 int nlist, int rs, int64_t cap, int4* __restrict__ items) {
    const int lane = threadIdx.x & 31;
    const int64_t l = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (l >= nlist) return;
    const int64_t a = item_off[l], b = item_off[l + 1];
    const int nrs = (list_size[l] + rs - 1) / rs;
    for (int64_t g = a + lane; g < b && g < cap; g += 32) {
        const int w = static_cast<int>(g - a);
        items[g] = make_int4(static_cast<int>(l), w / max(nrs, 1), w % max(nrs, 1), 0);
    }
}

// The inversion in two launches (nlist <= INVERT_SMEM_LISTS).  The first
// counts pairs per list in shared memory (each CTA a contiguous range of
// `per` pairs, loads in flight eight at a time) and adds the counts to
// w.pair_cnt; the last CTA to finish (a ticket on w.done after a fence)
// turns the counts into pair offsets and item offsets, zeroes the fill
// counters and resets the ticket.  The second places the pairs (as
// probe_fill_smem_kernel) and writes the item descriptors.
__device__ inline int64_t probe_list(const int64_t* __restrict__ probes, int64_t i, int wd, int nprobe, int j0) {
    return probes[(i / wd) * nprobe + j0 + i % wd];
}

__global__ void __launch_bounds__(512) invert_count_kernel(const int64_t* __restrict__ probes, int nq, int nprobe,
                                                           int j0, int j1, int nlist, int64_t per,
                                                           const int32_t* __restrict__ list_size, int rs, int qg,
                                                           BatchWork w) {
    extern __shared__ int h[];  // [nlist]
    __shared__ int s_last;
    __shared__ long long wpart[16];
    const int t = threadIdx.x;
    const int wd = j1 - j0;
    const int64_t n = static_cast<int64_t>(nq) * wd;
    const int64_t a = blockIdx.x * per, b = min(n, a + per);
    for (int l = t; l < nlist; l += blockDim.x) h[l] = 0;
    __syncthreads();
    for (int64_t i0 = a; i0 < b; i0 += 8 * 512) {
        int64_t l[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int64_t i = i0 + u * 512 + t;
            l[u] = i < b ? probe_list(probes, i, wd, nprobe, j0) : -1;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (l[u] >= 0) atomicAdd(&h[l[u]], 1);
    }
    __syncthreads();
    for (int l = t; l < nlist; l += blockDim.x)
        if (h[l]) atomicAdd(&w.pair_cnt[l], h[l]);
    __threadfence();
    __syncthreads();
    if (t == 0) s_last = atomicAdd(w.done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // Last CTA: pair offsets and item offsets (thread t: a contiguous run
    // of lists), fill counters zeroed, ticket reset.
    const int run = (nlist + 511) / 512;
    const int la = min(nlist, t * run), lb = min(nlist, la + run);
    long long sp = 0, si = 0;
    for (int l = la; l < lb; ++l) {
        const int c = __ldcg(&w.pair_cnt[l]), sz = list_size[l];
        sp += c;
        si += (c > 0 && sz > 0) ? static_cast<long long>((c + qg - 1) / qg) * ((sz + rs - 1) / rs) : 0;
        w.pair_fill[l] = 0;
    }
    // Two exclusive scans over the 512 runs (pairs, then items): within each
    // warp by shuffles, then over the 16 warp totals.
    const int lane = t & 31, warp = t >> 5;
    for (int pass = 0; pass < 2; ++pass) {
        const long long mine = pass == 0 ? sp : si;
        long long incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) wpart[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            long long x = lane < 16 ? wpart[lane] : 0;
#pragma unroll
            for (int o = 1; o < 16; o <<= 1) {
                const long long u = __shfl_up_sync(FULL, x, o);
                if (lane >= o) x += u;
            }
            if (lane < 16) wpart[lane] = x;  // inclusive over warps
        }
        __syncthreads();
        long long acc = incl - mine + (warp > 0 ? wpart[warp - 1] : 0);
        for (int l = la; l < lb; ++l) {
            const int c = __ldcg(&w.pair_cnt[l]), sz = list_size[l];
            if (pass == 0) {
                w.pair_off[l] = acc;
                acc += c;
            } else {
                w.item_off[l] = acc;
                acc += (c > 0 && sz > 0) ? static_cast<long long>((c + qg - 1) / qg) * ((sz + rs - 1) / rs) : 0;
            }
        }
        if (t == 511) {
            if (pass == 0)
                w.pair_off[nlist] = wpart[15];
            else
                w.item_off[nlist] = wpart[15];
        }
        __syncthreads();
    }
    if (t == 0) *w.done = 0u;
}

__global__ void __launch_bounds__(512) invert_fill_kernel(const int64_t* __restrict__ probes, int nq, int nprobe,
                                                          int j0, int j1, int nlist, int64_t per,
                                                          const int32_t* __restrict__ list_size, int rs,
                                                          BatchWork w) {
    extern __shared__ int h[];  // [nlist] counts, then ranks; [nlist] bases
    int* base = h + nlist;
    const int t = threadIdx.x;
    const int wd = j1 - j0;
    const int64_t n = static_cast<int64_t>(nq) * wd;
    const int64_t a = blockIdx.x * per, b = min(n, a + per);
    for (int l = t; l < nlist; l += blockDim.x) h[l] = 0;
    __syncthreads();
    for (int64_t i0 = a; i0 < b; i0 += 8 * 512) {
        int64_t l[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int64_t i = i0 + u * 512 + t;
            l[u] = i < b ? probe_list(probes, i, wd, nprobe, j0) : -1;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (l[u] >= 0) atomicAdd(&h[l[u]], 1);
    }
    __syncthreads();
    for (int l = t; l < nlist; l += blockDim.x) {
        base[l] = h[l] ? atomicAdd(&w.pair_fill[l], h[l]) : 0;
        h[l] = 0;
    }
    __syncthreads();
    for (int64_t i0 = a; i0 < b; i0 += 8 * 512) {
        int64_t l[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int64_t i = i0 + u * 512 + t;
            l[u] = i < b ? probe_list(probes, i, wd, nprobe, j0) : -1;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (l[u] >= 0) {
                const int64_t i = i0 + u * 512 + t;
                w.pairs[w.pair_off[l[u]] + base[l[u]] + atomicAdd(&h[l[u]], 1)] = static_cast<int32_t>(i / wd);
            }
    }
    // Item descriptors {list, query group, row slice} below item_cap, one
    // warp per list.
    const int lane = t & 31;
    for (int64_t l = blockIdx.x * 16 + (t >> 5); l < nlist; l += gridDim.x * 16) {
        const int64_t ia = w.item_off[l], ib = w.item_off[l + 1];
        const int nrs = max(1, (list_size[l] + rs - 1) / rs);
        for (int64_t g = ia + lane; g < ib && g < w.item_cap; g += 32) {
            const int k = static_cast<int>(g - ia);
            w.items[g] = make_int4(static_cast<int>(l), k / nrs, k % nrs, 0);
        }
    }
}

// ---------------------------------------------------------------------------
struct BatchedParams {
    const unsigned char* abf;       // tensor-core image of the arena (bf16 or e4m3)
    const int64_t* list_off;        // [nlist+1]
    const int32_t* list_size;       // [nlist]
    const int64_t* item_off;        // [nlist+1]
    const int4* items;              // [item_cap] {list, group, slice}
    int64_t item_cap;
    const int64_t* pair_off;        // [nlist+1]
    const int32_t* pairs;           // query ids grouped by list
    const int32_t* pair_cnt;        // [nlist]
    const float* xn;                // [arena rows] squared norms (f32)
    const float2* tile_aux;         // [arena tiles] {max |x~|, max |x - x~|} over the tile's rows
    const float2* xaux;             // [arena rows] {|x~|, |x - x~|} (dense items' error bounds)
    const unsigned char* qb;        // [nq][nkb*128 bytes] queries in the operand type
    const float4* qaux;             // [nq] {|q|^2, |q|, |q~|, |q - q~|}
    const float* lscale;            // e4m3 form: [nlist] list scales (x~ = lscale * code), else null
    const float* qscale;            // e4m3 form: [nq] query scales, else null
    const float* thr;               // [nq] distance thresholds (score units)
    uint64_t* cand;                 // [nq][capq]
    int32_t* cand_cnt;              // [nq]
    unsigned int* work;             // work-queue counter
    int* err;
    int nlist, nkb, rs, capq, metric;
    int ksplit;                     // 1: A k-blocks 2j, 2j+1 (hi, lo) both take query k-block j
    int ns;                         // stages in the list k-block ring (NS_MIN..NS_MAX)
    int nslot;                      // item slots (2 or SLOT_MAX)
    int dense_max;                  // lists of at most this many rows: dense items (0 = none)
    float cK, cN;                   // error-bound constants (see err_coef)
};

// Warp roles of the persistent batched kernel (12 warps).
constexpr int W_PRODUCER = 0;   // lane 0: bulk copies of list k-blocks
constexpr int W_MMA = 1;        // lane 0: tcgen05.mma issue; whole warp: TMEM alloc
constexpr int W_GATHER0 = 2;    // warps 2-3: fetch items, gather their queries
constexpr int N_GATHER = 2;
constexpr int W_EPI0 = 4;       // warps 4-11: epilogue (two per TMEM lane quadrant)
constexpr int N_EPI = 8;
constexpr int BATCH_THREADS = 32 * (W_EPI0 + N_EPI);
constexpr int CB = 256;         // per-epilogue-warp candidate staging

// Item metadata of one query slot.  Two slots hold the item being scanned and
// the next one being gathered; a third lets the gather run a further item
// ahead, since a slot only frees when the epilogue has finished its item.
constexpr int SLOT_MAX = 3;
constexpr int NS_SLOT3 = 5;   // three slots only when they leave this many stages
constexpr int RS_MAX = 2048;  // largest row slice (rows staged per slot)
template <int QG>
struct ItemSlot {
    int ntiles;  // -1 = no more items
    int nqv;
    int nrows;
    int lrow0;   // first row of the slice within its list
    int dense;   // 1: every row's score at its offset in the list, no threshold test
    long long row0;
    alignas(16) float xn[RS_MAX];  // |x|^2 of the slice's rows (cp.async target: 16-byte aligned)
    float2 taux[RS_MAX / TM];    // per tile {max |x~|, max |x - x~|}
    int qid[QG];
    float qn[QG];    // |q|^2
    float V[QG];     // threshold + bound constant - |q|^2 (score units)
    float aq[QG];    // bound coefficient of |x~|
    float bq[QG];    // bound coefficient of |x - x~|
    float cq[QG];    // bound constant
    alignas(16) float sc[QG];    // accumulator -> inner product scale (1, or list scale x query scale)
};

// Dynamic shared memory of the batched kernel for query groups of QG, nkb
// 128-byte k-blocks per row, ns stages and nslot item slots.
template <int QG>
constexpr size_t batched_smem(int nkb, int ns, int nslot) {
    constexpr int CW = QG / 2, CC = CW < 32 ? CW : 32;
    return 1024 + nslot * static_cast<size_t>(nkb) * QG * 128 + static_cast<size_t>(ns) * KB_BYTES +
           nslot * sizeof(ItemSlot<QG>) + N_EPI * CW * sizeof(float) + N_EPI * CB * (sizeof(int) + sizeof(uint64_t)) +
           N_EPI * 32 * CC * sizeof(float);
}
// Dynamic shared memory per CTA: the 227 KiB opt-in limit less room for the
// kernel's static shared variables (barriers, TMEM base, flags).
constexpr size_t BATCHED_SMEM_CAP = 227 * 1024 - 256;

// The deepest stage ring in [NS_MIN, NS_MAX] that fits (0: none fits).
template <int QG>
constexpr int batched_stages(int nkb, int nslot = 2) {
    for (int ns = NS_MAX; ns >= NS_MIN; --ns)
        if (batched_smem<QG>(nkb, ns, nslot) <= BATCHED_SMEM_CAP) return ns;
    return 0;
}

// Accumulator column of a group's i-th query (a bijection on [0, QG)).
template <int QG>
__device__ __forceinline__ int group_col(int i) {
    return (i >> 1) + (i & 1) * (QG / 2);
}

__device__ inline bool wait_or_abort(uint64_t* bar, uint32_t parity, int* err, volatile int* abort) {
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023u) == 1023u && *abort) return false;
    }
    if (err) atomicCAS(err, 0, DEV_ERR_TIMEOUT);
    *abort = 1;
    return false;
}

// Barrier over `nthreads` threads (a multiple of 32) on hardware barrier `id`.
__device__ inline void named_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// QG: queries per group (MMA N: 128, 64 or 32); F8: e4m3 operands
// (kind::f8f6f4, K = 32 per instruction) instead of bf16 (kind::f16, K = 16).
// Either way a k-block row is 128 bytes and one instruction covers 32 bytes
// of it, so the descriptors and the stage ring are the same.
template <int QG, bool F8>
__global__ void __launch_bounds__(BATCH_THREADS, 1) batched_scan_kernel(const __grid_constant__ BatchedParams p) {
    constexpr int CW = QG / 2;            // accumulator columns per epilogue warp
    constexpr int CC = CW < 32 ? CW : 32;  // columns per candidate-test chunk
    constexpr int TMEM_COLS = 2 * QG;      // two accumulators
    constexpr int BKB = QG * 128;          // bytes of one B (query) k-block
    using Slot = ItemSlot<QG>;
    extern __shared__ unsigned char sm_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
    const int nkb = p.nkb;                  // list (A) k-blocks per row
    const int nkbq = nkb >> p.ksplit;       // query (B) k-blocks per row
    const int nsl = p.nslot;                                         // item slots
    unsigned char* sB = base;                                        // nsl slots x nkb x BKB (queries)
    const int ns = p.ns;                                             // stages in the ring
    unsigned char* sA = sB + static_cast<size_t>(nsl) * nkbq * BKB;  // ns x 16 KiB (list k-blocks)
    Slot* slot = reinterpret_cast<Slot*>(sA + static_cast<size_t>(ns) * KB_BYTES);  // [nsl], 1024-aligned
    static_assert(offsetof(Slot, xn) % 16 == 0 && offsetof(Slot, sc) % 16 == 0 && sizeof(Slot) % 16 == 0,
                  "ItemSlot alignment");
    float* sR = reinterpret_cast<float*>(slot + nsl);                // [N_EPI][CW] per-tile test bounds
    int* s_cq = reinterpret_cast<int*>(sR + N_EPI * CW);             // [N_EPI][CB]
    uint64_t* s_ck = reinterpret_cast<uint64_t*>(s_cq + N_EPI * CB);  // [N_EPI][CB]
    float* s_ip = reinterpret_cast<float*>(s_ck + N_EPI * CB);       // [N_EPI][32 lanes][CC] candidate chunks

    __shared__ uint64_t full[NS_MAX], empty[NS_MAX], accf[2], acce[2], sfull[SLOT_MAX], sfree[SLOT_MAX];
    __shared__ uint32_t tbase;
    __shared__ int s_abort;
    __shared__ long long s_g[SLOT_MAX];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool l2 = p.metric == 1;
    volatile int* vabort = &s_abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < ns; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&accf[i], 1);
            mbar_init(&acce[i], N_EPI);
        }
        for (int i = 0; i < nsl; ++i) {
            mbar_init(&sfull[i], 32 * N_GATHER);
            mbar_init(&sfree[i], 1 + N_EPI);  // MMA commit + every epilogue warp
        }
        s_abort = 0;
        fence_mbar_init();
    }
    if (warp == W_MMA) tc::tmem_alloc(&tbase, TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;
    const int64_t total_items = p.item_off[p.nlist];

    if (warp >= W_GATHER0 && warp < W_GATHER0 + N_GATHER) {
        // ---------------- gather: fetch an item, decode it, stage its queries
        const int gt = threadIdx.x - 32 * W_GATHER0;  // 0..63
        for (uint32_t it = 0;; ++it) {
            const int b = static_cast<int>(it % nsl);
            if (!wait_or_abort(&sfree[b], ((it / nsl) & 1u) ^ 1u, p.err, vabort)) break;
            Slot& S = slot[b];
            // One index per slot: a gather thread may still be reading this
            // item's index while thread 0 already fetches the next one.
            if (gt == 0) s_g[b] = atomicAdd(p.work, 1u);
            named_sync(1, 32 * N_GATHER);
            const long long g = s_g[b];
            if (g >= total_items || *vabort) {
                if (gt == 0) S.ntiles = -1;
                mbar_arrive_cta(&sfull[b]);
                break;
            }
            int l, qg, rsl;
            if (g < p.item_cap) {
                const int4 d = p.items[g];
                l = d.x;
                qg = d.y;
                rsl = d.z;
            } else {
                // list = last l with item_off[l] <= g (lists without items
                // share the next list's offset and are skipped).
                int lo = 0, hi = p.nlist - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (p.item_off[mid] <= g)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                l = lo;
                const int w = static_cast<int>(g - p.item_off[l]);
                const int nrs = (p.list_size[l] + p.rs - 1) / p.rs;
                qg = w / nrs;
                rsl = w % nrs;
            }
            const int sz = p.list_size[l];
            const int nqv = min(QG, p.pair_cnt[l] - qg * QG);
            const int nrows = min(p.rs, sz - rsl * p.rs);
            const int32_t* grp = p.pairs + p.pair_off[l] + static_cast<int64_t>(qg) * QG;
            const long long row0 = p.list_off[l] + static_cast<long long>(rsl) * p.rs;
            const float ls = F8 ? p.lscale[l] : 1.0f;
            if (gt == 0) {
                S.nqv = nqv;
                S.nrows = nrows;
                S.lrow0 = rsl * p.rs;
                S.dense = sz <= p.dense_max;
                S.row0 = row0;
                S.ntiles = (nrows + TM - 1) / TM;
            }
            // A dense item: the list's first slice records each query's
            // entry count (the list size).
            if (sz <= p.dense_max && rsl == 0)
                for (int i = gt; i < nqv; i += 32 * N_GATHER) p.cand_cnt[grp[i]] = sz;
            // Row norms and tile bounds of the slice: asynchronous 16-byte
            // copies (the arena is padded to whole tiles, so the rounded-up
            // ranges stay inside it).
            for (int c = gt; c < (nrows + 3) / 4; c += 32 * N_GATHER) cp_async16(&S.xn[4 * c], p.xn + row0 + 4 * c);
            for (int c = gt; c < (nrows + TM - 1) / TM; c += 32 * N_GATHER) S.taux[c] = p.tile_aux[row0 / TM + c];
            // Query i of the group sits in accumulator column col(i): even
            // queries in the first half of the columns, odd ones in the
            // second, so a small group keeps both epilogue warps of every
            // TMEM lane quadrant busy.
            for (int i = gt; i < QG; i += 32 * N_GATHER) {
                const int col = group_col<QG>(i);
                const int qid = i < nqv ? grp[i] : -1;
                S.qid[col] = qid;
                if (qid >= 0) {
                    const float4 qa = p.qaux[qid];
                    const ErrCoef ec = err_coef(qa, l2, p.cK, p.cN);
                    S.qn[col] = l2 ? qa.x : 0.0f;
                    S.V[col] = p.thr[qid] + ec.cq - (l2 ? qa.x : 0.0f);
                    S.aq[col] = ec.aq;
                    S.bq[col] = ec.bq;
                    S.cq[col] = ec.cq;
                    S.sc[col] = F8 ? ls * p.qscale[qid] : 1.0f;
                } else {
                    S.qn[col] = 0.0f;
                    S.V[col] = -INFINITY;
                    S.aq[col] = 0.0f;
                    S.bq[col] = 0.0f;
                    S.cq[col] = 0.0f;
                    S.sc[col] = 0.0f;
                }
            }
            // The group's queries into the swizzled B operand (row = column
            // of the accumulator): every 16-byte chunk is its own
            // asynchronous copy, all in flight at once; empty query slots are
            // zero-filled.
            unsigned char* dst = sB + static_cast<size_t>(b) * nkbq * BKB;
            const size_t qstride = static_cast<size_t>(nkbq) * 128;
            for (int i = gt; i < QG; i += 32 * N_GATHER) {
                const int col = group_col<QG>(i);
                if (i < nqv) {
                    const unsigned char* src = p.qb + static_cast<size_t>(grp[i]) * qstride;
                    for (int kb = 0; kb < nkbq; ++kb)
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            cp_async16(dst + kb * BKB + col * 128 + (((c ^ (col & 7)) & 7) << 4),
                                       src + kb * 128 + c * 16);
                } else {
                    for (int kb = 0; kb < nkbq; ++kb)
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            *reinterpret_cast<uint4*>(dst + kb * BKB + col * 128 + (c << 4)) = make_uint4(0, 0, 0, 0);
                }
            }
            cp_async_wait_all();
            fence_proxy_async();  // generic-proxy writes -> tensor-core reads
            mbar_arrive_cta(&sfull[b]);
        }
    } else if (warp == W_PRODUCER) {
        // ---------------- producer: list k-blocks into the stage ring
        if (lane == 0) {
            int ls = 0;        // stage of the next copy
            uint32_t lph = 0;  // its ring round's parity
            for (uint32_t it = 0;; ++it) {
                const int b = static_cast<int>(it % nsl);
                if (!wait_or_abort(&sfull[b], (it / nsl) & 1u, p.err, vabort)) break;
                const int ntiles = slot[b].ntiles;
                if (ntiles < 0) break;
                const int64_t tile0 = slot[b].row0 / TM;
                bool ok = true;
                for (int t = 0; t < ntiles && ok; ++t) {
                    for (int kb = 0; kb < nkb; ++kb) {
                        const int s = ls;
                        const uint32_t ph = lph;
                        if (++ls == ns) {
                            ls = 0;
                            lph ^= 1u;
                        }
                        if (!wait_or_abort(&empty[s], ph ^ 1u, p.err, vabort)) {
                            ok = false;
                            break;
                        }
                        mbar_expect_tx(&full[s], KB_BYTES);
                        bulk_g2s(sA + static_cast<size_t>(s) * KB_BYTES,
                                 p.abf + ((tile0 + t) * nkb + kb) * static_cast<int64_t>(KB_BYTES), KB_BYTES,
                                 &full[s]);
                    }
                }
                if (!ok) break;
            }
        }
    } else if (warp == W_MMA) {
        // ---------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = F8 ? tc::idesc_e4m3_f32(TM, QG) : tc::idesc_bf16_f32(TM, QG);
            int ms = 0;        // stage of the next k-block
            uint32_t mph = 0;  // its ring round's parity
            uint32_t tile_it = 0;
            bool ok = true;
            for (uint32_t it = 0; ok; ++it) {
                const int b = static_cast<int>(it % nsl);
                if (!wait_or_abort(&sfull[b], (it / nsl) & 1u, p.err, vabort)) break;
                const int ntiles = slot[b].ntiles;
                if (ntiles < 0) break;
                tc::fence_after_sync();
                const uint32_t b0 = smem_u32(sB + static_cast<size_t>(b) * nkbq * BKB);
                for (int t = 0; t < ntiles && ok; ++t, ++tile_it) {
                    const int buf = tile_it & 1;
                    if (!wait_or_abort(&acce[buf], ((tile_it >> 1) & 1u) ^ 1u, p.err, vabort)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t dcol = tmem + static_cast<uint32_t>(buf * QG);
                    for (int kb = 0; kb < nkb; ++kb) {
                        const int s = ms;
                        const uint32_t ph = mph;
                        if (++ms == ns) {
                            ms = 0;
                            mph ^= 1u;
                        }
                        if (!wait_or_abort(&full[s], ph, p.err, vabort)) {
                            ok = false;
                            break;
                        }
                        tc::fence_after_sync();
                        const uint32_t a0 = smem_u32(sA + static_cast<size_t>(s) * KB_BYTES);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            const uint64_t ad = tc::sdesc_sw128(a0 + kk * 32);
                            const uint64_t bd = tc::sdesc_sw128(b0 + (kb >> p.ksplit) * BKB + kk * 32);
                            if constexpr (F8)
                                tc::mma_e4m3(dcol, ad, bd, idesc, (kb | kk) != 0 ? 1u : 0u);
                            else
                                tc::mma_bf16(dcol, ad, bd, idesc, (kb | kk) != 0 ? 1u : 0u);
                        }
                        tc::mma_commit(&empty[s]);
                    }
                    if (ok) tc::mma_commit(&accf[buf]);
                }
                if (ok) tc::mma_commit(&sfree[b]);  // the slot's queries are no longer read
            }
        }
    } else if (warp >= W_EPI0) {
        // ---------------- epilogue: thread = row of the tile; each warp of a
        // TMEM lane quadrant handles half of the QG query columns.
        const int e = warp - W_EPI0;       // 0..7
        const int quad = warp & 3;         // TMEM lanes [32*quad, 32*quad+32)
        const int half = e >> 2;           // columns [CW*half, CW*half+CW)
        int* wq = s_cq + e * CB;
        uint64_t* wk = s_ck + e * CB;
        // Candidate staging: a ring of CB entries in NSEG segments; wc counts
        // every candidate this warp staged (warp-uniform, in a register).
        // When the fill crosses into a new segment, the segment just filled
        // reserves its buffer slots (one counter atomic per entry, results
        // kept in registers) and the oldest reserved segment, which the fill
        // is about to overwrite, stores its entries: the atomics' latency
        // overlaps the emission of the next segments.
        constexpr int NSEG = 4, SEG = CB / NSEG, SJ = SEG / 32;
        int wc = 0, npend = 0;
        int pos0[SJ], pos1[SJ], pos2[SJ];  // reserved slots, oldest .. newest
        auto reserve = [&](int seg, int n, int (&pos)[SJ]) {
#pragma unroll
            for (int j = 0; j < SJ; ++j) {
                const int i = lane + 32 * j;
                pos[j] = i < n ? atomicAdd(&p.cand_cnt[wq[seg * SEG + i]], 1) : p.capq;
            }
        };
        auto store = [&](int seg, const int (&pos)[SJ]) {
#pragma unroll
            for (int j = 0; j < SJ; ++j) {
                const int i = seg * SEG + lane + 32 * j;
                if (pos[j] < p.capq) p.cand[static_cast<int64_t>(wq[i]) * p.capq + pos[j]] = wk[i];
            }
        };
        const float cf = l2 ? -2.0f : -1.0f;
        uint32_t tile_it = 0;
        for (uint32_t it = 0;; ++it) {
            const int b = static_cast<int>(it % nsl);
            if (!wait_or_abort(&sfull[b], (it / nsl) & 1u, p.err, vabort)) break;
            const Slot& S = slot[b];
            const int ntiles = S.ntiles;
            if (ntiles < 0) break;
            // Occupied columns of this warp's half: [0, nact) of its CW.
            const int nact = (S.nqv + 1 - half) >> 1;
            const int nrows = S.nrows;
            const long long row0 = S.row0;
            bool ok = true;
            float* R = sR + e * CW;  // this warp's CW columns
            for (int t = 0; t < ntiles; ++t, ++tile_it) {
                const int buf = tile_it & 1;
                // Per-tile test bound of this warp's queries:
                // V + max|x~| aq + max|x - x~| bq over the tile's rows.
                const float2 ta = S.taux[t];
                __syncwarp();
                for (int cc = lane; cc < CW; cc += 32) {
                    const int q = half * CW + cc;
                    R[cc] = S.V[q] + fmaf(ta.x, S.aq[q], ta.y * S.bq[q]);
                }
                __syncwarp();
                if (!wait_or_abort(&accf[buf], (tile_it >> 1) & 1u, p.err, vabort)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const int rs_row = t * TM + quad * 32 + lane;
                const bool rvalid = rs_row < nrows;
                const long long arow = row0 + rs_row;
                const float xnv = rvalid ? S.xn[rs_row] : 0.0f;
                // Rows past the slice end compare as NaN: never candidates.
                const float ax = rvalid ? (l2 ? xnv - err_row_const(xnv, l2, p.cN) : 0.0f) : __int_as_float(0x7fffffff);
                // This warp's occupied columns in one TMEM load (the first
                // chunk alone when the rest are empty); the accumulator is
                // released to the MMA warp right after it.
                uint32_t u[CW];
                const uint32_t taddr =
                    tmem + (static_cast<uint32_t>(quad * 32) << 16) + static_cast<uint32_t>(buf * QG + half * CW);
                if constexpr (CW > CC) {
                    if (nact <= CC) {
                        uint32_t u0[CC];
                        tc::tmem_ld_cols<CC>(taddr, u0);
#pragma unroll
                        for (int j = 0; j < CC; ++j) u[j] = u0[j];
#pragma unroll
                        for (int j = CC; j < CW; ++j) u[j] = 0u;
                    } else {
                        tc::tmem_ld_cols<CW>(taddr, u);
                    }
                } else {
                    tc::tmem_ld_cols<CW>(taddr, u);
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive_cta(&acce[buf]);
                if (S.dense) {
                    // Dense item: every valid row of every occupied column
                    // writes its score (4 bytes) at the row's offset in the
                    // list within the upper half of the query's buffer (the
                    // warp's 32 rows are 128 contiguous bytes); the threshold
                    // is not consulted, and the tightening step recomputes
                    // each row's error bound from the row's terms.
                    const int pos = S.lrow0 + rs_row;
                    if (rvalid && pos < p.capq) {
                        float* cfs = reinterpret_cast<float*>(p.cand) + p.capq;
#pragma unroll
                        for (int j = 0; j < CW; ++j) {
                            if (j >= nact) break;
                            const int q = half * CW + j;
                            const float ip = F8 ? __uint_as_float(u[j]) * S.sc[q] : __uint_as_float(u[j]);
                            const float score = l2 ? __fadd_rn(__fadd_rn(xnv, S.qn[q]), -2.0f * ip) : -ip;
                            cfs[static_cast<int64_t>(S.qid[q]) * (2 * p.capq) + pos] = score;
                        }
                    }
                    continue;
                }
#pragma unroll
                for (int c = 0; c < CW / CC; ++c) {
                    const int col0 = half * CW + c * CC;
                    if (c * CC >= nact) continue;
                    // The chunk's test bounds (and, for e4m3, the
                    // accumulator scales) in registers.
                    float r[CC], m[CC];
#pragma unroll
                    for (int j = 0; j < CC; j += 4) {
                        const float4 t4 = *reinterpret_cast<const float4*>(R + c * CC + j);
                        r[j] = t4.x;
                        r[j + 1] = t4.y;
                        r[j + 2] = t4.z;
                        r[j + 3] = t4.w;
                        if constexpr (F8) {
                            const float4 m4 = *reinterpret_cast<const float4*>(S.sc + col0 + j);
                            m[j] = cf * m4.x;
                            m[j + 1] = cf * m4.y;
                            m[j + 2] = cf * m4.z;
                            m[j + 3] = cf * m4.w;
                        } else {
                            m[j] = m[j + 1] = m[j + 2] = m[j + 3] = cf;
                        }
                    }
                    // candidate test: cf*ip + (|x|^2 - cx) <= R_q (see err_coef).
                    // First only whether any row of the warp has one in the
                    // chunk (two instructions per element); the per-column
                    // mask is built for such chunks alone.
                    bool hit = false;
#pragma unroll
                    for (int j = 0; j < CC; ++j) hit |= fmaf(m[j], __uint_as_float(u[c * CC + j]), ax) <= r[j];
                    if (!__any_sync(FULL, hit)) continue;
                    uint32_t mask = 0;
#pragma unroll
                    for (int j = 0; j < CC; ++j)
                        mask |= (fmaf(m[j], __uint_as_float(u[c * CC + j]), ax) <= r[j]) ? (1u << j) : 0u;
                    const unsigned cols = __reduce_or_sync(FULL, mask);
                    if (cols) {
                        // Some rows of the warp have candidates in the chunk.
                        // Their accumulators go to private shared-memory rows;
                        // then, column by column (warp-uniform), the lanes with
                        // a candidate there write it at their ballot rank.
                        float* sip = s_ip + (e * 32 + lane) * CC;
                        if (mask) {
#pragma unroll
                            for (int j = 0; j < CC; j += 4)
                                *reinterpret_cast<float4*>(sip + j) =
                                    make_float4(__uint_as_float(u[c * CC + j]), __uint_as_float(u[c * CC + j + 1]),
                                                __uint_as_float(u[c * CC + j + 2]), __uint_as_float(u[c * CC + j + 3]));
                        }
                        unsigned left = cols;
                        while (left) {
                            const int j = __ffs(left) - 1;
                            left &= left - 1u;
                            const bool mine = (mask >> j) & 1u;
                            const unsigned bal = __ballot_sync(FULL, mine);
                            const int cnt = __popc(bal);
                            const bool cross = (wc + cnt) / SEG != wc / SEG;  // warp-uniform
                            if (cross && npend == NSEG - 1) {
                                // The segment about to be refilled: its slots
                                // were reserved three crossings ago.
                                store((wc / SEG + 1) % NSEG, pos0);
                                --npend;
                                __syncwarp();
                            }
                            if (mine) {
                                const int q = col0 + j;
                                const float ip = F8 ? sip[j] * S.sc[q] : sip[j];
                                const float score = l2 ? __fadd_rn(__fadd_rn(xnv, S.qn[q]), -2.0f * ip) : -ip;
                                const int at = (wc + __popc(bal & ((1u << lane) - 1u))) & (CB - 1);
                                wq[at] = S.qid[q];
                                wk[at] = (static_cast<uint64_t>(f2o(score)) << 32) | static_cast<uint32_t>(arow);
                            }
                            if (cross) {
                                __syncwarp();
#pragma unroll
                                for (int j = 0; j < SJ; ++j) {
                                    pos0[j] = pos1[j];
                                    pos1[j] = pos2[j];
                                }
                                reserve((wc / SEG) % NSEG, SEG, pos2);
                                ++npend;
                            }
                            wc += cnt;
                        }
                    }
                }
            }
            if (lane == 0) mbar_arrive_cta(&sfree[b]);
            if (!ok) break;
        }
        // Drain: the reserved segments, then the partly filled one.
        const int last = (wc / SEG + NSEG - 1) % NSEG;  // newest reserved segment
        if (npend >= 3) store((last + NSEG - 2) % NSEG, pos0);
        if (npend >= 2) store((last + NSEG - 1) % NSEG, pos1);
        if (npend >= 1) store(last, pos2);
        __syncwarp();
        int posr[SJ];
        reserve((wc / SEG) % NSEG, wc % SEG, posr);
        store((wc / SEG) % NSEG, posr);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == W_MMA) tc::tmem_dealloc(tmem, TMEM_COLS);
}

// ---------------------------------------------------------------------------
// Threshold tightening between the two batched passes.  Each candidate's
// exact distance lies in [s - e, s + e], so U = the k-th smallest s + e over a
// query's candidates bounds its final k-th distance from above:
// thr := min(thr, U), and candidates with s - e > U can never enter the top-k
// and are dropped from the buffer (kept ones are compacted to its front).  A
// query whose buffer already overflowed is left untouched so the re-rank still
// reports it.
constexpr int TIGHTEN_PER_THREAD = 48;  // 256 threads x 48 >= the largest capq (12288)

__global__ void __launch_bounds__(256) tighten_kernel(const float* __restrict__ xn, const float2* __restrict__ xaux,
                                                      const float4* __restrict__ qaux, BatchWork w, int capq, int k,
                                                      int metric, float cK, float cN, float* __restrict__ thr) {
    extern __shared__ __align__(16) unsigned char sm[];
    uint32_t* hi = reinterpret_cast<uint32_t*>(sm);  // [capq]
    float* lo = reinterpret_cast<float*>(hi + capq);  // [capq]
    __shared__ int hist[256];
    __shared__ uint32_t sh[2];
    __shared__ int s_m;
    const bool l2 = metric == 1;
    // Queries left by the warp kernel (w.big2: count, then ids), a CTA each.
    const int nbig = w.big2[0];
    for (int li = blockIdx.x; li < nbig; li += gridDim.x) {
    const int qi = w.big2[1 + li];
    __syncthreads();  // the previous query's shared state is no longer read
    const int cnt = w.cand_cnt[qi];
    if (cnt < k || cnt > capq) continue;
    const int n = cnt;
    uint64_t* cq = w.cand + static_cast<int64_t>(qi) * capq;
    const ErrCoef ec = err_coef(qaux[qi], l2, cK, cN);
    // Keys stay in registers (element i = threadIdx.x + 256 t) so the buffer
    // can be compacted in place after every thread has read it.
    uint64_t kr[TIGHTEN_PER_THREAD];
#pragma unroll
    for (int t = 0; t < TIGHTEN_PER_THREAD; ++t) {
        const int i = threadIdx.x + 256 * t;
        kr[t] = 0;
        if (i < n) {
            const uint64_t key = cq[i];
            const int64_t row = static_cast<int64_t>(key & 0xffffffffu);
            const float2 xa = xaux[row];
            const float e = fmaf(xa.x, ec.aq, fmaf(xa.y, ec.bq, err_row_const(xn[row], l2, cN) + ec.cq));
            const float sc = o2f(static_cast<uint32_t>(key >> 32));
            kr[t] = key;
            hi[i] = f2o(sc + e);
            lo[i] = sc - e;
        }
    }
    if (threadIdx.x == 0) s_m = 0;
    __syncthreads();
    int need;
    const float U = o2f(cta_radix_select(hi, n, k, &need, hist, sh));
#pragma unroll
    for (int t = 0; t < TIGHTEN_PER_THREAD; ++t) {
        const int i = threadIdx.x + 256 * t;
        if (i < n && lo[i] <= U) cq[atomicAdd(&s_m, 1)] = kr[t];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        w.cand_cnt[qi] = s_m;
        if (U < thr[qi]) thr[qi] = U;
    }
    }
}

// Warp tighten of one query with k <= cnt <= 32 * PER candidates (PER per
// lane in registers).
template <int PER>
__device__ inline void tighten_warp_query(int qi, int cnt, const float* __restrict__ xn,
                                          const float2* __restrict__ xaux, const float4* __restrict__ qaux,
                                          const BatchWork& w, int capq, int k, bool l2, float cK, float cN,
                                          float* __restrict__ thr, int* hist, int lane) {
    const ErrCoef ec = err_coef(qaux[qi], l2, cK, cN);
    uint64_t* cq = w.cand + static_cast<int64_t>(qi) * capq;
    uint32_t hi[PER];
    float lo[PER];
#pragma unroll
    for (int r = 0; r < PER; ++r) {
        const int e = r * 32 + lane;
        hi[r] = 0xffffffffu;
        lo[r] = INFINITY;
        if (e < cnt) {
            const uint64_t key = cq[e];
            const int64_t row = static_cast<int64_t>(key & 0xffffffffu);
            const float2 xa = xaux[row];
            const float eb = fmaf(xa.x, ec.aq, fmaf(xa.y, ec.bq, err_row_const(xn[row], l2, cN) + ec.cq));
            const float sc = o2f(static_cast<uint32_t>(key >> 32));
            hi[r] = f2o(sc + eb);
            lo[r] = sc - eb;
        }
    }
    const float U = o2f(warp_select_bound<PER>(hi, cnt, k, hist, lane));
    // In-place compaction of the candidates that can still enter the top-k:
    // every element of a round is read before any of that round's writes.
    int m = 0;
#pragma unroll
    for (int r = 0; r < PER; ++r) {
        const int e = r * 32 + lane;
        const bool keep = e < cnt && lo[r] <= U;
        const uint64_t key = e < cnt ? cq[e] : 0;
        const unsigned b = __ballot_sync(FULL, keep);
        __syncwarp();
        if (keep) cq[m + __popc(b & ((1u << lane) - 1u))] = key;
        m += __popc(b);
    }
    if (lane == 0) {
        w.cand_cnt[qi] = m;
        if (U < thr[qi]) thr[qi] = U;
    }
}

// An upper bound U on the k-th smallest score + bound of cnt >= k
// {score, bound} entries (get(e) gives entry e), with at least k entries at
// or below it: two 8-bit radix passes below the bits all the entries'
// ordered values share; U is the upper edge of the final bin that holds the
// k-th value.  One warp; the entries are read on every pass.
template <typename Get>
__device__ inline float kth_bound_stream(Get get, int cnt, int k, int* hist, int lane) {
    uint32_t mn = 0xffffffffu, mx = 0u;
#pragma unroll 8
    for (int e = lane; e < cnt; e += 32) {
        const float2 v = get(e);
        const uint32_t h = f2o(v.x + v.y);
        mn = min(mn, h);
        mx = max(mx, h);
    }
    mn = __reduce_min_sync(FULL, mn);
    mx = __reduce_max_sync(FULL, mx);
    uint32_t ub = mn;
    if (mn != mx) {
        // Two 8-bit radix passes below the bits every value shares.
        int top = 31 - __clz(mn ^ mx);
        uint32_t mask = ~((2u << top) - 1u);
        uint32_t prefix = mn & mask;
        int rem = k;
#pragma unroll 1
        for (int pass = 0; pass < 2 && top >= 0; ++pass) {
            const int shift = top > 7 ? top - 7 : 0;
            const uint32_t wmask = ((2u << top) - 1u) & ~((1u << shift) - 1u);
#pragma unroll
            for (int i = 0; i < 8; ++i) hist[lane * 8 + i] = 0;
            __syncwarp();
#pragma unroll 8
            for (int e = lane; e < cnt; e += 32) {
                const float2 v = get(e);
                const uint32_t h = f2o(v.x + v.y);
                if ((h & mask) == prefix) atomicAdd(&hist[(h & wmask) >> shift], 1);
            }
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
            int digit = lane * 8 + 7, before = excl;
            if (mine) {
                int cum = excl;
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
            const int src = __ffs(__ballot_sync(FULL, mine)) - 1;
            digit = __shfl_sync(FULL, digit, src);
            before = __shfl_sync(FULL, before, src);
            prefix |= static_cast<uint32_t>(digit) << shift;
            mask |= wmask;
            rem -= before;
            top = shift - 1;
            __syncwarp();
        }
        ub = top >= 0 ? (prefix | ((2u << top) - 1u)) : prefix;
    }
    return o2f(ub);
}

// k-th bound of a dense first-pass buffer in one read, held in registers:
// lane l reads entries l, l + 32, ... (entry(e) = {score, bound}), four at a
// time, and keeps the M smallest upper values (score + bound) it sees: the
// four are sorted and merged into the kept M (the elementwise minimum of
// the kept values and the four reversed is a bitonic sequence holding the M
// smallest, which a bitonic merge sorts).  U is then an upper bound on the
// k-th smallest of the 32*M kept values (32*M >= k): the kept values'
// k-th, searched bit by bit over 16 bits below the bits they all share, and
// the upper edge of the final bin.  Every kept value is an entry's, so at
// least k entries lie at or below U; values were only left out, so U is at
// or above the k-th smallest upper value of the whole buffer.  With
// cnt >= k every lane keeps all its entries or M of them, so the k-th kept
// value is an entry's, never the padding (0xffffffff).
template <int M, typename Entry>
__device__ inline float dense_kth_regs(Entry entry, int cnt, int k, int lane) {
    static_assert(M >= 4 && (M & (M - 1)) == 0, "M: a power of two, at least 4");
    auto cx = [](uint32_t& x, uint32_t& y) {
        const uint32_t lo = min(x, y);
        y = max(x, y);
        x = lo;
    };
    uint32_t a[M];
#pragma unroll
    for (int i = 0; i < M; ++i) a[i] = 0xffffffffu;
    for (int e0 = lane; e0 < cnt; e0 += 128) {
        uint32_t b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = e0 + 32 * i;
            b[i] = 0xffffffffu;
            if (e < cnt) {
                const float2 v = entry(e);
                b[i] = f2o(v.x + v.y);
            }
        }
        cx(b[0], b[1]);
        cx(b[2], b[3]);
        cx(b[0], b[2]);
        cx(b[1], b[3]);
        cx(b[1], b[2]);
#pragma unroll
        for (int i = 0; i < 4; ++i) a[M - 4 + i] = min(a[M - 4 + i], b[3 - i]);
#pragma unroll
        for (int st = M / 2; st > 0; st >>= 1)
#pragma unroll
            for (int i = 0; i < M; ++i)
                if ((i & st) == 0) cx(a[i], a[i + st]);
    }
    const uint32_t mn = __reduce_min_sync(FULL, a[0]);
    const uint32_t mx = __reduce_max_sync(FULL, a[M - 1]);
    if (mn == mx) return o2f(mn);
    const int top = 31 - __clz(mn ^ mx);
    const int low = top > 15 ? top - 15 : 0;
    uint32_t R = mn & ~((2u << top) - 1u);
#pragma unroll 1
    for (int bit = top; bit >= low; --bit) {
        const uint32_t T = R | ((1u << bit) - 1u);
        int c = 0;
#pragma unroll
        for (int i = 0; i < M; ++i) c += a[i] <= T ? 1 : 0;
        if (static_cast<int>(__reduce_add_sync(FULL, static_cast<unsigned>(c))) < k) R |= 1u << bit;
    }
    return o2f(R | ((1u << low) - 1u));
}

// Warp tighten of a query whose first-pass list was scanned densely: the
// upper half of its buffer holds cnt scores, entry i for row i of the list
// (arena rows from row0); each entry's error bound is recomputed from the
// row's {|x~|, |x - x~|} and squared norm and the query's coefficients,
// the same expression as the batched kernel's candidate test.  U = an upper
// bound on the k-th smallest score + bound with at least k entries at or
// below it (dense_kth_regs); the entries with score - bound <= U are
// rewritten as keys (score, arena row) at the front of the buffer (key m
// overwrites bytes [8m, 8m + 8), below every entry not yet read, which sit
// at 4 capq + 4e with e >= m).  Fewer than k entries: every entry is kept
// and the threshold is left alone.
__device__ inline void tighten_dense_query(int qi, int cnt, int64_t row0, const float* __restrict__ xn,
                                           const float2* __restrict__ xaux, const float4* __restrict__ qaux,
                                           const float2* __restrict__ tile_aux, const float* __restrict__ tile_xn,
                                           bool l2, float cK, float cN, const BatchWork& w, int capq, int k,
                                           float* __restrict__ thr, int lane) {
    uint64_t* cq = w.cand + static_cast<int64_t>(qi) * capq;
    const float* cs = reinterpret_cast<const float*>(cq) + capq;
    const ErrCoef ec = err_coef(qaux[qi], l2, cK, cN);
    // B = the bound expression at the list's tile maxima of |x~|, |x - x~|
    // and |x|^2: every row's bound is at most B (each rounded operation is
    // monotone in its non-negative operands).
    float mx = 0.0f, my = 0.0f, mn = 0.0f;
    for (int64_t t = row0 / TM + lane; t < (row0 + cnt + TM - 1) / TM; t += 32) {
        const float2 a = tile_aux[t];
        mx = fmaxf(mx, a.x);
        my = fmaxf(my, a.y);
        mn = fmaxf(mn, tile_xn[t]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
        my = fmaxf(my, __shfl_xor_sync(FULL, my, o));
        mn = fmaxf(mn, __shfl_xor_sync(FULL, mn, o));
    }
    const float B = fmaf(mx, ec.aq, fmaf(my, ec.bq, err_row_const(mn, l2, cN) + ec.cq));
    // U = (k-th smallest score) + B: at least k entries have score + bound
    // at or below it.
    float U = INFINITY;
    auto score = [&](int e) { return make_float2(cs[e], 0.0f); };
    // M about twice k/32: a lane reads more than M of the k smallest rarely.
    if (cnt >= k)
        U = (k <= 32    ? dense_kth_regs<4>(score, cnt, k, lane)
             : k <= 128 ? dense_kth_regs<8>(score, cnt, k, lane)
                        : dense_kth_regs<16>(score, cnt, k, lane)) +
            B;
    // An entry is kept when score - bound <= U: at once when score <= U,
    // never when score - B > U, else with the row's own bound.
    const float2* xa = xaux + row0;
    const float* xr = xn + row0;
    auto keep_entry = [&](float sc, int e) {
        if (sc <= U) return true;
        if (sc - B > U) return false;
        const float2 a = xa[e];
        return sc - fmaf(a.x, ec.aq, fmaf(a.y, ec.bq, err_row_const(xr[e], l2, cN) + ec.cq)) <= U;
    };
    // In-place rewrite, four rounds of 32 at a time: all four rounds are
    // read (loads in flight together) before any of their writes, and writes
    // never pass the reads.
    int m = 0;
    for (int base = 0; base < cnt; base += 128) {
        float v[4];
        bool kp[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = base + 32 * i + lane;
            v[i] = e < cnt ? cs[e] : 0.0f;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = base + 32 * i + lane;
            kp[i] = e < cnt && keep_entry(v[i], e);
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = base + 32 * i + lane;
            const unsigned b = __ballot_sync(FULL, kp[i]);
            if (kp[i])
                cq[m + __popc(b & ((1u << lane) - 1u))] =
                    (static_cast<uint64_t>(f2o(v[i])) << 32) | static_cast<uint32_t>(row0 + e);
            m += __popc(b);
        }
    }
    if (lane == 0) {
        w.cand_cnt[qi] = m;
        if (U < thr[qi]) thr[qi] = U;
    }
}

// Warp tighten: one warp per query with at most 1024 candidates (or a dense
// first-pass list of any size); buffers of up to 2048 go to
// tighten_warp2_kernel through w.big, larger ones to the CTA kernel through
// w.big2.
constexpr int TIGHTEN_WARP_MAX = 1024;

__global__ void __launch_bounds__(256) tighten_warp_kernel(const float* __restrict__ xn,
                                                           const float2* __restrict__ xaux,
                                                           const float4* __restrict__ qaux, int nq, BatchWork w,
                                                           int capq, int k, int metric, float cK, float cN,
                                                           float* __restrict__ thr, DenseFirst df) {
    __shared__ int hist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto one = [&](int qi) {
        const int cnt = w.cand_cnt[qi];
        if (cnt < k) return;
        if (cnt > capq) return;  // overflowed: left for the re-rank to report
        if (cnt > TIGHTEN_WARP_MAX) {
            if (lane == 0) {
                if (cnt > 2 * TIGHTEN_WARP_MAX)
                    w.big2[1 + atomicAdd(&w.big2[0], 1)] = qi;
                else
                    w.big[1 + atomicAdd(&w.big[0], 1)] = qi;
            }
            return;
        }
        tighten_warp_query<TIGHTEN_WARP_MAX / 32>(qi, cnt, xn, xaux, qaux, w, capq, k, metric == 1, cK, cN, thr,
                                                  hist[warp], lane);
    };
    if (df.dense_max > 0) {
        // The queries tighten_dense_kernel listed (first-pass list not dense).
        const int n = w.rest[0];
        for (int li = blockIdx.x * 8 + warp; li < n; li += gridDim.x * 8) one(w.rest[1 + li]);
        return;
    }
    for (int qi = blockIdx.x * 8 + warp; qi < nq; qi += gridDim.x * 8) one(qi);
}

// Queries whose first-pass list was scanned densely, one warp each.
__global__ void __launch_bounds__(256) tighten_dense_kernel(const float* __restrict__ xn,
                                                            const float2* __restrict__ xaux,
                                                            const float4* __restrict__ qaux, int nq, BatchWork w,
                                                            int capq, int k, int metric, float cK, float cN,
                                                            float* __restrict__ thr, DenseFirst df) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * 8 + warp;
    if (qi >= nq) return;  // whole warp
    const int64_t l0 = df.probes[static_cast<int64_t>(qi) * df.nprobe];
    if (l0 < 0 || df.list_size[l0] > df.dense_max) {
        // Thresholded first-pass list: tighten_warp_kernel's.
        if (lane == 0) w.rest[1 + atomicAdd(&w.rest[0], 1)] = qi;
        return;
    }
    tighten_dense_query(qi, w.cand_cnt[qi], df.list_off[l0], xn, xaux, qaux, df.tile_aux, df.tile_xn, metric == 1, cK,
                        cN, w, capq, k, thr, lane);
}

// Queries with 1025..2048 candidates (w.big), one warp each.
__global__ void __launch_bounds__(256) tighten_warp2_kernel(const float* __restrict__ xn,
                                                            const float2* __restrict__ xaux,
                                                            const float4* __restrict__ qaux, BatchWork w, int capq,
                                                            int k, int metric, float cK, float cN,
                                                            float* __restrict__ thr) {
    __shared__ int hist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nbig = w.big[0];
    for (int li = blockIdx.x * 8 + warp; li < nbig; li += gridDim.x * 8) {
        const int qi = w.big[1 + li];
        tighten_warp_query<2 * TIGHTEN_WARP_MAX / 32>(qi, w.cand_cnt[qi], xn, xaux, qaux, w, capq, k, metric == 1,
                                                      cK, cN, thr, hist[warp], lane);
    }
}

// ---------------------------------------------------------------------------
// The coarse quantiser on the tensor cores.  The centroids form a one-list
// index of their own (rows padded to whole 128-row tiles with zeros): its
// split bf16 image, per-row bound terms, squared norms (the sequential f32
// sum the arena's rows get) and per-tile maxima.  Split image: each value c
// as hi = bf16(c) and lo = bf16(c - hi); a tile holds, per 64 dimensions,
// the hi k-block then the lo k-block, and the batched kernel multiplies
// both by the same query k-block, so the accumulator sums q~.(hi + lo)
// (|c - hi - lo| <= 2^-16 |c|, against 2^-8 |c| for one bf16).  Bound terms
// {|(|hi| + |lo|)|, |c - hi - lo|}: the first covers |hi + lo| and the
// magnitudes the accumulation adds.
__global__ void rowmajor_image_kernel(const float* __restrict__ x, int64_t n, int d, int nkb, int64_t rows,
                                      unsigned char* __restrict__ out) {
    const int w = nkb * 64;
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= rows * w) return;
    const int64_t r = i / w;
    const int j = static_cast<int>(i % w);
    const float v = (r < n && j < d) ? x[r * d + j] : 0.0f;
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    const uint32_t off = tc::kblock_offset(static_cast<uint32_t>(r & 127), j & 63);
    unsigned char* tile = out + (r >> 7) * (2 * nkb) * KB_BYTES;
    *reinterpret_cast<__nv_bfloat16*>(tile + (2 * (j >> 6)) * KB_BYTES + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(tile + (2 * (j >> 6) + 1) * KB_BYTES + off) = lo;
}

__global__ void rowmajor_aux_kernel(const float* __restrict__ x, int64_t n, int d, int64_t rows,
                                    float2* __restrict__ aux, float* __restrict__ xn) {
    const int lane = threadIdx.x & 31;
    const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (r >= rows) return;
    float nn = 0.0f, ee = 0.0f;
    if (r < n)
        for (int j = lane; j < d; j += 32) {
            const float v = x[r * d + j];
            const float hi = __bfloat162float(__float2bfloat16_rn(v));
            const float lo = __bfloat162float(__float2bfloat16_rn(v - hi));
            const float m = fabsf(hi) + fabsf(lo);
            const float e = (v - hi) - lo;  // exact: both differences are of nearby values
            nn = fmaf(m, m, nn);
            ee = fmaf(e, e, ee);
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nn += __shfl_xor_sync(FULL, nn, o);
        ee += __shfl_xor_sync(FULL, ee, o);
    }
    if (lane == 0) {
        float sq = 0.0f;
        if (r < n)
            for (int j = 0; j < d; ++j) sq = __fadd_rn(sq, __fmul_rn(x[r * d + j], x[r * d + j]));
        aux[r] = make_float2(sqrtf(nn), sqrtf(ee));
        xn[r] = sq;
    }
}

// Work of one coarse launch: every query in the centroid list's groups, each
// group split into nslices row slices.
__global__ void coarse_items_kernel(int nq, int nlist, int64_t rows, int ngroups, int nslices,
                                    int64_t* __restrict__ list_off, int32_t* __restrict__ list_size, BatchWork w) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t nitems = static_cast<int64_t>(ngroups) * nslices;
    if (i < nq) w.pairs[i] = static_cast<int32_t>(i);
    if (i < nitems) w.items[i] = make_int4(0, static_cast<int>(i / nslices), static_cast<int>(i % nslices), 0);
    if (i == 0) {
        list_off[0] = 0;
        list_off[1] = rows;
        list_size[0] = nlist;
        w.pair_cnt[0] = nq;
        w.pair_off[0] = 0;
        w.pair_off[1] = nq;
        w.item_off[0] = 0;
        w.item_off[1] = nitems;
    }
}

// Staging row pitch of coarse_refine_kernel (floats): d + 4 when d is a
// multiple of 4 (16-byte rows), else d + 1 (conflict-free column reads).
__host__ __device__ inline int refine_pitch(int d) { return (d & 3) == 0 ? d + 4 : d + 1; }
// Shared memory per warp of the refine kernels: the copy barrier (16 bytes
// with padding), 256 histogram bins, the query and a 32-row staging block.
__host__ __device__ inline size_t refine_warp_bytes(int d) {
    const size_t pitch = refine_pitch(d);
    return (16 + 1024 + pitch * 4 + 32 * pitch * 4 + 15) & ~size_t(15);
}

// Exact coarse selection from the tensor-core scores.  Per query (one warp):
// the upper half of cand holds nlist scores; with each centroid's error
// bound recomputed from its {|c~|, |c - c~|} and squared norm and the
// query's coefficients, the {score, bound} pairs are held in registers (PER
// per lane); U = an upper bound on the m-th smallest score + bound
// (warp_select_bound); every centroid whose score - bound <= U (a set that
// holds the exact m best, ties included) gets its exact FP32 coarse score
// with the same sequential arithmetic as coarse_scores_kernel (dimension
// order, separately rounded operations), and the m best (score, centroid)
// keys, ascending with ties to the lower centroid, are written as
// select_warp_kernel writes them.  The candidate keys overwrite the query's
// pairs in cand.  Shared memory per warp: the copy barrier, 256 histogram
// bins, the query and a 32-row staging block of centroids.
// The exact m best of a query's c candidate centroids (ids in keys[0, c),
// and in sids[0, c) when sids is given and c <= 256): exact FP32 coarse
// scores with coarse_scores_kernel's arithmetic (dimension order, separately
// rounded operations), 32 candidates per round (lane i sums row i), then
// ordered by (score, centroid) and written as select_warp_kernel writes them.
// With d a multiple of 4 the rows are staged in shared memory (row pitch
// d + 4, so a warp's 512-byte read takes the minimum four wavefronts), each
// lane's row by one bulk copy completing on a barrier (the cost of a bulk
// copy is per copy, not per byte: whole rows measured faster than
// dimension halves pipelined against the sums).  Up to 128 candidates the scored keys stay in
// registers (lane i, round r: candidate 32 r + i); more are written back to
// keys and merged through shared-memory-free warp sorts.
template <int METRIC>
__device__ inline float coarse_dot(const float* qs, const float* row, int j0, int j1, float acc) {
#pragma unroll 4
    for (int jj = j0; jj < j1; jj += 4) {
        const float4 a = *reinterpret_cast<const float4*>(qs + jj);
        const float4 b = *reinterpret_cast<const float4*>(row + jj);
        if (METRIC == METRIC_L2) {
            acc = sq_add(acc, a.x, b.x);
            acc = sq_add(acc, a.y, b.y);
            acc = sq_add(acc, a.z, b.z);
            acc = sq_add(acc, a.w, b.w);
        } else {
            acc = ip_add(acc, a.x, b.x);
            acc = ip_add(acc, a.y, b.y);
            acc = ip_add(acc, a.z, b.z);
            acc = ip_add(acc, a.w, b.w);
        }
    }
    return acc;
}

// Ranks of a warp's c <= 32 R keys (lane i, round r: key 32 r + i in kr[r],
// all c of them also in kbuf) among one another, and each of the m smallest
// written at its rank.
template <int R>
__device__ inline void rank_write(const uint64_t (&kr)[4], const uint64_t* kbuf, int c, int m, int qi,
                                  int64_t* __restrict__ out_idx, float* __restrict__ out_score, int lane) {
    int rank[R];
#pragma unroll
    for (int i = 0; i < R; ++i) rank[i] = 0;
    int e = 0;
    for (; e + 1 < c; e += 2) {
        const ulonglong2 two = *reinterpret_cast<const ulonglong2*>(kbuf + e);
#pragma unroll
        for (int i = 0; i < R; ++i) rank[i] += (two.x < kr[i] ? 1 : 0) + (two.y < kr[i] ? 1 : 0);
    }
    if (e < c) {
        const uint64_t one = kbuf[e];
#pragma unroll
        for (int i = 0; i < R; ++i) rank[i] += one < kr[i] ? 1 : 0;
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
        if (i * 32 + lane < c && rank[i] < m) {
            out_idx[static_cast<int64_t>(qi) * m + rank[i]] = static_cast<int64_t>(kr[i] & 0xffffffffu);
            if (out_score) out_score[static_cast<int64_t>(qi) * m + rank[i]] = o2f(static_cast<uint32_t>(kr[i] >> 32));
        }
    }
}

template <int METRIC>
__device__ inline void coarse_exact_best(uint64_t* keys, const int* sids, uint64_t* kbuf, uint64_t* bars, int c,
                                         const float* qs, float* stage, int pitch, const float* __restrict__ cent,
                                         int d, int m, int qi, int64_t* __restrict__ out_idx,
                                         float* __restrict__ out_score, int* err, int lane) {
    // Fewer candidates than m (not reached when the bound holds m of them):
    // the missing probes are -1.
    for (int e = c + lane; e < m; e += 32) {
        out_idx[static_cast<int64_t>(qi) * m + e] = -1;
        if (out_score) out_score[static_cast<int64_t>(qi) * m + e] = FLT_MAX;
    }
    const bool v4 = (d & 3) == 0;
    const bool in_regs = c <= 128;
    const bool ids_smem = sids != nullptr && c <= 256;
    auto cid_of = [&](int e) { return ids_smem ? sids[e] : static_cast<int>(keys[e]); };
    uint64_t kr[4] = {KEY_MAX, KEY_MAX, KEY_MAX, KEY_MAX};
    if (v4) {
        const uint32_t rb = static_cast<uint32_t>(d) * 4u;  // bytes of one row
        uint64_t* bar = &bars[0];
        if (lane == 0) {
            mbar_init(bar, 1);
            fence_mbar_init();
        }
        __syncwarp();
        uint32_t issued = 0, used = 0;  // phases of the barrier issued and consumed
        // nr rows: lane i's row (centroid cid_) by one bulk copy completing
        // on the barrier.  A round's reads of the staging block have all
        // returned (every lane's sum used them before the __syncwarp that
        // precedes the next round's copies), as in a copy pipeline whose
        // consumers release a stage by arriving on a barrier.
        auto copy_rows = [&](int cid_, int nr) {
            if (lane == 0) mbar_expect_tx(bar, static_cast<uint32_t>(nr) * rb);
            __syncwarp();
            if (lane < nr) bulk_g2s(stage + lane * pitch, cent + static_cast<size_t>(cid_) * d, rb, bar);
            ++issued;
        };
        int cid = lane < min(32, c) ? cid_of(lane) : 0;
        if (c > 0) copy_rows(cid, min(32, c));
        bool ok = true;
        for (int c0 = 0, r = 0; c0 < c; c0 += 32, ++r) {
            const int nr = min(32, c - c0);
            const int nn = max(0, min(32, c - c0 - 32));  // next round's rows
            const int cidn = lane < nn ? cid_of(c0 + 32 + lane) : 0;
            float acc = 0.0f;
            ok = mbar_wait_bounded(bar, used & 1u, err);
            if (!ok) break;
            ++used;
            if (lane < nr) acc = coarse_dot<METRIC>(qs, stage + lane * pitch, 0, d, acc);
            __syncwarp();
            if (nn) copy_rows(cidn, nn);
            if (lane < nr) {
                const float score = METRIC == METRIC_L2 ? acc : -acc;
                const uint64_t key = (static_cast<uint64_t>(f2o(score)) << 32) | static_cast<uint32_t>(cid);
                if (in_regs) {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (i == r) kr[i] = key;
                } else {
                    keys[c0 + lane] = key;
                }
            }
            cid = cidn;
        }
        if (!ok) {
            // A copy that did not complete in time: the status word is
            // raised; wait (bounded) for whatever is still in flight, and
            // write nothing.
            while (used < issued && mbar_wait_bounded(bar, used & 1u, nullptr)) ++used;
            return;
        }
        __syncwarp();
    } else {
        for (int c0 = 0, r = 0; c0 < c; c0 += 32, ++r) {
            const int nr = min(32, c - c0);
            const int cidr = lane < nr ? cid_of(c0 + lane) : 0;
            for (int rr = 0; rr < nr; ++rr) {
                const float* src = cent + static_cast<size_t>(__shfl_sync(FULL, cidr, rr)) * d;
                float* dst = stage + rr * pitch;
                for (int j = lane; j < d; j += 32) cp_async4(dst + j, src + j);
            }
            cp_async_wait_all();
            __syncwarp();
            if (lane < nr) {
                const float* row = stage + lane * pitch;
                float acc = 0.0f;
                for (int jj = 0; jj < d; ++jj)
                    acc = METRIC == METRIC_L2 ? sq_add(acc, qs[jj], row[jj]) : ip_add(acc, qs[jj], row[jj]);
                const float score = METRIC == METRIC_L2 ? acc : -acc;
                const uint64_t key = (static_cast<uint64_t>(f2o(score)) << 32) | static_cast<uint32_t>(cidr);
                if (in_regs) {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (i == r) kr[i] = key;
                } else {
                    keys[c0 + lane] = key;
                }
            }
            __syncwarp();
        }
    }
    // The m smallest keys, ascending.  Up to 128 candidates: each key's rank
    // is the number of smaller keys (keys are distinct: the centroid is in
    // the low bits), and it goes to that position.  The keys are read back
    // as shared-memory broadcasts, two per load.
    if (in_regs) {
        __syncwarp();  // the candidate ids (which kbuf may overlay) are read
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r * 32 + lane < c) kbuf[r * 32 + lane] = kr[r];
        __syncwarp();
        switch ((c + 31) >> 5) {
            case 1: rank_write<1>(kr, kbuf, c, m, qi, out_idx, out_score, lane); break;
            case 2: rank_write<2>(kr, kbuf, c, m, qi, out_idx, out_score, lane); break;
            case 3: rank_write<3>(kr, kbuf, c, m, qi, out_idx, out_score, lane); break;
            case 4: rank_write<4>(kr, kbuf, c, m, qi, out_idx, out_score, lane); break;
            default: break;
        }
        return;
    }
    __syncwarp();
    // More: sorted blocks of 256 merged into the running best 256.
    uint64_t t[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int e = r * 32 + lane;
        t[r] = e < c ? keys[e] : KEY_MAX;
    }
    warp_sort<8>(t, lane);
    for (int c0 = 256; c0 < c; c0 += 256) {
        uint64_t u[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int e = c0 + r * 32 + lane;
            u[r] = e < c ? keys[e] : KEY_MAX;
        }
        warp_sort<8>(u, lane);
        warp_merge<8>(t, u, lane);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int e = r * 32 + lane;
        if (e < m && e < c) {
            out_idx[static_cast<int64_t>(qi) * m + e] = static_cast<int64_t>(t[r] & 0xffffffffu);
            if (out_score) out_score[static_cast<int64_t>(qi) * m + e] = o2f(static_cast<uint32_t>(t[r] >> 32));
        }
    }
}

template <int METRIC, int PER>
__global__ void __launch_bounds__(128, 1) coarse_refine_kernel(float2* __restrict__ cand, int nq, int nlist,
                                                            const float* __restrict__ q,
                                                            const float* __restrict__ cent,
                                                            const float* __restrict__ cxn,
                                                            const float2* __restrict__ caux,
                                                            const float4* __restrict__ qaux, float cK, float cN,
                                                            int d, int m, int64_t* __restrict__ out_idx,
                                                            float* __restrict__ out_score, int* err) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pitch = refine_pitch(d);
    unsigned char* base = sm + warp * refine_warp_bytes(d);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base);
    int* hist = reinterpret_cast<int*>(base + 16);
    float* qs = reinterpret_cast<float*>(hist + 256);
    float* stage = qs + pitch;
    const int qi = blockIdx.x * (blockDim.x >> 5) + warp;
    if (qi >= nq) return;  // whole warp
    const float* qrow = q + static_cast<size_t>(qi) * d;
    for (int j = lane; j < d; j += 32) qs[j] = qrow[j];
    // Every centroid's upper bound (ordered bits) and lower bound in
    // registers: entry r * 32 + lane, or, with exactly 32 PER centroids,
    // entry 4 (32 (r / 4) + lane) + r % 4 (16-byte loads of four centroids'
    // terms).  The query's buffer is then free and holds its candidate keys.
    float2* ce = cand + static_cast<int64_t>(qi) * nlist;
    const float* cs = reinterpret_cast<const float*>(ce) + nlist;
    uint64_t* keys = reinterpret_cast<uint64_t*>(ce);
    const bool l2 = METRIC == METRIC_L2;
    const ErrCoef ec = err_coef(qaux[qi], l2, cK, cN);
    const bool vec = nlist == PER * 32;
    auto entry = [&](int r) { return vec ? 4 * ((r >> 2) * 32 + lane) + (r & 3) : r * 32 + lane; };
    uint32_t hi[PER];
    float lo[PER];
    auto bound = [&](int r, float sc, float ax, float ay, float xn) {
        const float eb = fmaf(ax, ec.aq, fmaf(ay, ec.bq, err_row_const(xn, l2, cN) + ec.cq));
        hi[r] = f2o(sc + eb);
        lo[r] = sc - eb;
    };
    if (vec) {
#pragma unroll
        for (int g = 0; g < PER / 4; ++g) {
            const int e0 = 4 * (g * 32 + lane);
            const float4 sc = *reinterpret_cast<const float4*>(cs + e0);
            const float4 a01 = *reinterpret_cast<const float4*>(caux + e0);
            const float4 a23 = *reinterpret_cast<const float4*>(caux + e0 + 2);
            const float4 xn = *reinterpret_cast<const float4*>(cxn + e0);
            bound(4 * g, sc.x, a01.x, a01.y, xn.x);
            bound(4 * g + 1, sc.y, a01.z, a01.w, xn.y);
            bound(4 * g + 2, sc.z, a23.x, a23.y, xn.z);
            bound(4 * g + 3, sc.w, a23.z, a23.w, xn.w);
        }
    } else {
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int e = r * 32 + lane;
            hi[r] = 0xffffffffu;
            lo[r] = INFINITY;
            if (e < nlist) bound(r, cs[e], caux[e].x, caux[e].y, cxn[e]);
        }
    }
    const float U = o2f(warp_select_bound<PER>(hi, nlist, m, hist, lane));
    __syncwarp();  // every pair has been read, and the histogram too
    // Centroids that can be among the m best: the first 256 ids in the
    // histogram's space, the rest in keys (and there all of them when there
    // are more than 256).
    int c = 0;
#pragma unroll
    for (int r = 0; r < PER; ++r) {
        const int e = entry(r);
        const bool keep = e < nlist && lo[r] <= U;
        const unsigned bal = __ballot_sync(FULL, keep);
        if (keep) {
            const int at = c + __popc(bal & ((1u << lane) - 1u));
            if (at < 256)
                hist[at] = e;
            else
                keys[at] = static_cast<uint64_t>(e);
        }
        c += __popc(bal);
    }
    __syncwarp();
    if (c > 256)
        for (int e = lane; e < 256; e += 32) keys[e] = static_cast<uint64_t>(hist[e]);
    __syncwarp();
    coarse_exact_best<METRIC>(keys, hist, reinterpret_cast<uint64_t*>(hist), bars, c, qs, stage, pitch, cent, d, m,
                              qi, out_idx, out_score, err, lane);
}

// The coarse step for more than 2048 lists, in two tensor-core launches.
// First a dense launch over the first S centroids; coarse_thr_kernel takes
// each query's bound on the m-th smallest score + bound among them, which
// bounds its m-th best exact coarse score over all centroids from above.
// Then a thresholded launch over all centroids emits the (score, centroid)
// keys whose lower bound reaches it, and coarse_refine_keys_kernel selects
// and re-scores them exactly.
__global__ void __launch_bounds__(256) coarse_thr_kernel(const float2* __restrict__ cand, int nq, int S, int m,
                                                         const float* __restrict__ cxn,
                                                         const float2* __restrict__ caux,
                                                         const float4* __restrict__ qaux, int metric, float cK,
                                                         float cN, float* __restrict__ thr) {
    __shared__ int hist[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * 8 + warp;
    if (qi >= nq) return;  // whole warp
    // The dense launch's scores (upper half of the query's buffer) and each
    // centroid's recomputed error bound.
    const float* cs = reinterpret_cast<const float*>(cand + static_cast<int64_t>(qi) * S) + S;
    const bool l2 = metric == METRIC_L2;
    const ErrCoef ec = err_coef(qaux[qi], l2, cK, cN);
    uint32_t hv[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        const int e = r * 32 + lane;
        hv[r] = 0xffffffffu;
        if (e < S) {
            const float2 a = caux[e];
            const float eb = fmaf(a.x, ec.aq, fmaf(a.y, ec.bq, err_row_const(cxn[e], l2, cN) + ec.cq));
            hv[r] = f2o(cs[e] + eb);
        }
    }
    const float U = o2f(warp_select_bound<32>(hv, S, m, hist[warp], lane));
    if (lane == 0) thr[qi] = U;
}

// Per query (one warp): its n keys (score, centroid) at cand + qi * stride;
// every key's bound from the centroid's {|c~|, |c - c~|} and squared norm and
// the query's coefficients; U = an upper bound on the m-th smallest
// score + bound; the centroids with score - bound <= U go to
// coarse_exact_best.
template <int METRIC>
__global__ void __launch_bounds__(128, 1) coarse_refine_keys_kernel(uint64_t* __restrict__ cand,
                                                                 const int32_t* __restrict__ ccnt, int nq, int stride,
                                                                 const float* __restrict__ q,
                                                                 const float* __restrict__ cent,
                                                                 const float* __restrict__ cxn,
                                                                 const float2* __restrict__ caux,
                                                                 const float4* __restrict__ qaux, int d, int m,
                                                                 float cK, float cN, int64_t* __restrict__ out_idx,
                                                                 float* __restrict__ out_score, int* err) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pitch = refine_pitch(d);
    unsigned char* base = sm + warp * refine_warp_bytes(d);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base);
    int* hist = reinterpret_cast<int*>(base + 16);
    float* qs = reinterpret_cast<float*>(hist + 256);
    float* stage = qs + pitch;
    const int qi = blockIdx.x * (blockDim.x >> 5) + warp;
    if (qi >= nq) return;  // whole warp
    const float* qrow = q + static_cast<size_t>(qi) * d;
    for (int j = lane; j < d; j += 32) qs[j] = qrow[j];
    const bool l2 = METRIC == METRIC_L2;
    const ErrCoef ec = err_coef(qaux[qi], l2, cK, cN);
    uint64_t* keys = cand + static_cast<int64_t>(qi) * stride;
    const int n = min(ccnt[qi], stride);
    auto get = [&](int e) {
        const uint64_t kk = keys[e];
        const uint32_t row = static_cast<uint32_t>(kk & 0xffffffffu);
        const float2 xa = caux[row];
        const float eb = fmaf(xa.x, ec.aq, fmaf(xa.y, ec.bq, err_row_const(cxn[row], l2, cN) + ec.cq));
        return make_float2(o2f(static_cast<uint32_t>(kk >> 32)), eb);
    };
    const float U = n >= m ? kth_bound_stream(get, n, m, hist, lane) : INFINITY;
    // In place: the kept centroids' ids to the front (every element of a
    // round is read before any of that round's writes).
    int c = 0;
    for (int b0 = 0; b0 < n; b0 += 32) {
        const int e = b0 + lane;
        bool keep = false;
        uint64_t id = 0;
        if (e < n) {
            const float2 v = get(e);
            keep = v.x - v.y <= U;
            id = keys[e] & 0xffffffffu;
        }
        const unsigned bal = __ballot_sync(FULL, keep);
        __syncwarp();
        if (keep) keys[c + __popc(bal & ((1u << lane) - 1u))] = id;
        c += __popc(bal);
    }
    __syncwarp();
    coarse_exact_best<METRIC>(keys, nullptr, reinterpret_cast<uint64_t*>(hist), bars, c, qs, stage, pitch, cent, d,
                              m, qi, out_idx, out_score, err, lane);
}

// ---------------------------------------------------------------------------
// Exact re-rank.  Every candidate carries its bf16 distance s and error bound
// e (recomputed from the row and query quantities), so its exact distance
// lies in [s - e, s + e].  U = the k-th smallest s + e bounds the query's
// exact k-th distance from above; only candidates with s - e <= U can belong
// to the exact top-k, and those get their exact FP32 distance (the plain
// scan's arithmetic).  The k best (distance, arena row) keys are written as
// (D, I).  A query whose candidate buffer or re-rank set overflowed is listed
// in w.overflow for the caller.
constexpr int RERANK_MAX = 4096;

// Warp re-rank of one query with at most KR*32 candidates, all in registers
// (element e = r*32 + lane): U = the k-th smallest upper bound s + e (warp
// bitonic sort), the selected set = candidates with s - e <= U (for rmax > 0
// only the rmax with the smallest s), their exact FP32 distances (the plain
// scan's arithmetic, spread over the lanes through the warp's shared list
// sl), a final sort, the top k written out.
template <int KR>
__device__ void rerank_warp_query(const ArenaLayout& L, const float* __restrict__ codes,
                                  const int64_t* __restrict__ ids, const float* __restrict__ xn,
                                  const float2* __restrict__ xaux, const ErrCoef& ec, const uint64_t* cq, int n, int k,
                                  int rmax, bool l2, float cN, bool exact, const float* qs, uint64_t* sl,
                                  float* __restrict__ Dq, int64_t* __restrict__ Iq, int lane) {
    uint64_t key[KR], srt[KR];
    if (exact && rmax == 0) {
        // Certified exact tensor-core distances: the k smallest keys
        // (distance, arena row) are the answer, the same ones the bounded
        // selection below would keep.
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const int e = r * 32 + lane;
            srt[r] = e < n ? cq[e] : KEY_MAX;
        }
        warp_sort<KR>(srt, lane);
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const int e = r * 32 + lane;
            if (e < k) {
                const uint64_t kk = srt[r];
                if (kk == KEY_MAX) {
                    Dq[e] = l2 ? FLT_MAX : -FLT_MAX;
                    Iq[e] = -1;
                } else {
                    const float sc = o2f(static_cast<uint32_t>(kk >> 32));
                    Dq[e] = l2 ? sc : -sc;
                    Iq[e] = ids[kk & 0xffffffffu];
                }
            }
        }
        return;
    }
    float lo[KR];
#pragma unroll
    for (int r = 0; r < KR; ++r) {
        const int e = r * 32 + lane;
        key[r] = KEY_MAX;
        srt[r] = KEY_MAX;
        lo[r] = INFINITY;
        if (e < n) {
            const uint64_t kk = cq[e];
            const int64_t row = static_cast<int64_t>(kk & 0xffffffffu);
            const float sc = o2f(static_cast<uint32_t>(kk >> 32));
            const float2 xa = xaux[row];
            const float eb = fmaf(xa.x, ec.aq, fmaf(xa.y, ec.bq, err_row_const(xn[row], l2, cN) + ec.cq));
            key[r] = kk;
            lo[r] = sc - eb;
            srt[r] = static_cast<uint64_t>(f2o(sc + eb)) << 32;
        }
    }
    float U = INFINITY;
    if (n > k) {
        warp_sort<KR>(srt, lane);
        U = o2f(static_cast<uint32_t>(warp_get<KR>(srt, k - 1) >> 32));
    }
    bool sel[KR];
    int nsel = 0;
#pragma unroll
    for (int r = 0; r < KR; ++r) {
        sel[r] = key[r] != KEY_MAX && lo[r] <= U;
        nsel += sel[r] ? 1 : 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nsel += __shfl_xor_sync(FULL, nsel, o);
    if (rmax > 0 && nsel > rmax) {
#pragma unroll
        for (int r = 0; r < KR; ++r) srt[r] = sel[r] ? key[r] : KEY_MAX;
        warp_sort<KR>(srt, lane);
        const uint32_t Sr = static_cast<uint32_t>(warp_get<KR>(srt, rmax - 1) >> 32);
#pragma unroll
        for (int r = 0; r < KR; ++r) sel[r] = sel[r] && static_cast<uint32_t>(key[r] >> 32) <= Sr;
    }
    if (exact) {
        // Certified exact tensor-core distances: the selected keys are final.
#pragma unroll
        for (int r = 0; r < KR; ++r) srt[r] = sel[r] ? key[r] : KEY_MAX;
    } else {
        int m = 0;
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const unsigned b = __ballot_sync(FULL, sel[r]);
            if (sel[r]) sl[m + __popc(b & ((1u << lane) - 1u))] = key[r] & 0xffffffffu;
            m += __popc(b);
        }
        __syncwarp();
        for (int i = lane; i < m; i += 32) {
            const int64_t row = static_cast<int64_t>(sl[i]);
            const float sc = l2 ? row_l2_global(L, codes, row, qs, true) : -row_ip_global(L, codes, row, qs);
            sl[i] = (static_cast<uint64_t>(f2o(sc)) << 32) | static_cast<uint32_t>(row);
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const int e = r * 32 + lane;
            srt[r] = e < m ? sl[e] : KEY_MAX;
        }
    }
    warp_sort<KR>(srt, lane);
#pragma unroll
    for (int r = 0; r < KR; ++r) {
        const int e = r * 32 + lane;
        if (e < k) {
            const uint64_t kk = srt[r];
            if (kk == KEY_MAX) {
                Dq[e] = l2 ? FLT_MAX : -FLT_MAX;
                Iq[e] = -1;
            } else {
                const float sc = o2f(static_cast<uint32_t>(kk >> 32));
                Dq[e] = l2 ? sc : -sc;
                Iq[e] = ids[kk & 0xffffffffu];
            }
        }
    }
}

// One warp per query; a query with more than 256 candidates (or k > 256, or
// an overflowed buffer) is listed in w.big for the CTA kernel.  (Capping the
// register sorts at 256 keys keeps the kernel at 64 registers: four CTAs per
// SM.)
__global__ void __launch_bounds__(256) rerank_warp_kernel(const __grid_constant__ ArenaLayout L,
                                                          const float* __restrict__ codes,
                                                          const int64_t* __restrict__ ids, const float* __restrict__ xn,
                                                          const float2* __restrict__ xaux,
                                                          const float4* __restrict__ qaux, const float* __restrict__ q,
                                                          int nq, BatchWork w, int capq, int k, int rmax, int metric,
                                                          float cK, float cN, const int32_t* __restrict__ qexact,
                                                          float* __restrict__ D, int64_t* __restrict__ I) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t* sl = reinterpret_cast<uint64_t*>(sm) + static_cast<size_t>(warp) * 256;  // [8][256] selected keys
    float* qs = reinterpret_cast<float*>(reinterpret_cast<uint64_t*>(sm) + 8 * 256) +
                static_cast<size_t>(warp) * L.row_pitch;
    const int qi = blockIdx.x * 8 + warp;
    if (qi >= nq) return;  // whole warp
    const int cnt = w.cand_cnt[qi];
    const int n = min(cnt, capq);
    if (cnt > capq || n > 256 || k > 256) {
        if (lane == 0) w.big[1 + atomicAdd(&w.big[0], 1)] = qi;
        return;
    }
    const float* src = q + static_cast<size_t>(qi) * L.d;
    for (int i = lane; i < L.row_pitch; i += 32) {
        int b = 0;
        while (b + 1 < L.nb && i >= L.boff[b + 1]) ++b;
        const int j = i - L.boff[b];
        qs[i] = j < L.bstart[b + 1] - L.bstart[b] ? src[L.bstart[b] + j] : 0.0f;
    }
    __syncwarp();
    const bool l2 = metric == 1;
    const ErrCoef ec = err_coef(qaux[qi], l2, cK, cN);
    const uint64_t* cq = w.cand + static_cast<int64_t>(qi) * capq;
    float* Dq = D + static_cast<size_t>(qi) * k;
    int64_t* Iq = I + static_cast<size_t>(qi) * k;
    const int need = max(n, k);
    const bool exact = qexact != nullptr && qexact[qi] != 0;
    if (need <= 128)
        rerank_warp_query<4>(L, codes, ids, xn, xaux, ec, cq, n, k, rmax, l2, cN, exact, qs, sl, Dq, Iq, lane);
    else
        rerank_warp_query<8>(L, codes, ids, xn, xaux, ec, cq, n, k, rmax, l2, cN, exact, qs, sl, Dq, Iq, lane);
}

__global__ void __launch_bounds__(256) rerank_kernel(ArenaLayout L, const float* __restrict__ codes,
                                                     const int64_t* __restrict__ ids, const float* __restrict__ xn,
                                                     const float2* __restrict__ xaux, const float4* __restrict__ qaux,
                                                     const float* __restrict__ q, BatchWork w, int qbase, int capq,
                                                     int k, int rmax, int metric, float cK, float cN,
                                                     const int32_t* __restrict__ qexact, float* __restrict__ D,
                                                     int64_t* __restrict__ I) {
    extern __shared__ __align__(16) unsigned char sm[];
    uint64_t* sel = reinterpret_cast<uint64_t*>(sm);                  // [RERANK_MAX]
    float* qs = reinterpret_cast<float*>(sel + RERANK_MAX);           // [row_pitch]
    uint32_t* hi = reinterpret_cast<uint32_t*>(qs + L.row_pitch);     // [capq] ordered s + e
    float* lo = reinterpret_cast<float*>(hi + capq);                  // [capq] s - e
    __shared__ int hist[256];
    __shared__ uint32_t sh[2];
    __shared__ int s_nsel, s_over;
    const bool l2 = metric == 1;
    // Queries left by the warp re-rank (w.big: count, then ids), a CTA each.
    const int nbig = w.big[0];
    for (int li = blockIdx.x; li < nbig; li += gridDim.x) {
    const int qi = w.big[1 + li];
    __syncthreads();  // the previous query's shared state is no longer read
    const int cnt = w.cand_cnt[qi];
    const int n = min(cnt, capq);
    const uint64_t* cq = w.cand + static_cast<int64_t>(qi) * capq;
    const float4 qa = qaux[qi];
    const ErrCoef ec = err_coef(qa, l2, cK, cN);
    if (threadIdx.x == 0) {
        s_nsel = 0;
        s_over = cnt > capq ? 1 : 0;
    }
    stage_query(L, q + static_cast<size_t>(qi) * L.d, qs);
    // Certified exact tensor-core distances need no bounds (e = 0).
    const bool no_bounds = qexact != nullptr && qexact[qi] != 0 && rmax == 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t key = cq[i];
        const int64_t row = static_cast<int64_t>(key & 0xffffffffu);
        const float sc = o2f(static_cast<uint32_t>(key >> 32));
        float e = 0.0f;
        if (!no_bounds) {
            const float2 xa = xaux[row];
            e = fmaf(xa.x, ec.aq, fmaf(xa.y, ec.bq, err_row_const(xn[row], l2, cN) + ec.cq));
        }
        hi[i] = f2o(sc + e);
        lo[i] = sc - e;
    }
    __syncthreads();
    float U = INFINITY;
    if (n > k) {
        int need;
        U = o2f(cta_radix_select(hi, n, k, &need, hist, sh));
    }
    // Oversampled re-rank (rmax > 0): of the candidates whose bound can reach
    // the top-k, only the rmax with the smallest tensor-core distance.
    uint32_t Sr = 0xffffffffu;
    if (rmax > 0 && n > rmax) {
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            hi[i] = lo[i] <= U ? static_cast<uint32_t>(cq[i] >> 32) : 0xffffffffu;
        __syncthreads();
        int need;
        Sr = cta_radix_select(hi, n, rmax, &need, hist, sh);
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (lo[i] <= U && static_cast<uint32_t>(cq[i] >> 32) <= Sr) {
            const int pos = atomicAdd(&s_nsel, 1);
            if (pos < RERANK_MAX)
                sel[pos] = cq[i];
            else
                s_over = 1;
        }
    }
    __syncthreads();
    const int m = min(s_nsel, RERANK_MAX);
    if (threadIdx.x == 0 && s_over) {
        const int pos = atomicAdd(&w.overflow[0], 1);
        w.overflow[1 + pos] = qbase + qi;
    }
    const bool exact = qexact != nullptr && qexact[qi] != 0;  // certified exact keys need no recompute
    for (int i = threadIdx.x; i < m && !exact; i += blockDim.x) {
        const int64_t row = static_cast<int64_t>(sel[i] & 0xffffffffu);
        const float sc = l2 ? row_l2_global(L, codes, row, qs, true) : -row_ip_global(L, codes, row, qs);
        sel[i] = (static_cast<uint64_t>(f2o(sc)) << 32) | static_cast<uint32_t>(row);
    }
    const int P = next_pow2(max(m, 1));
    for (int i = m + threadIdx.x; i < P; i += blockDim.x) sel[i] = KEY_MAX;
    __syncthreads();
    cta_bitonic_sort(sel, P);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const uint64_t key = i < m ? sel[i] : KEY_MAX;
        float dv;
        int64_t iv;
        if (key == KEY_MAX) {
            dv = l2 ? FLT_MAX : -FLT_MAX;
            iv = -1;
        } else {
            const float sc = o2f(static_cast<uint32_t>(key >> 32));
            dv = l2 ? sc : -sc;
            iv = ids[key & 0xffffffffu];
        }
        D[static_cast<size_t>(qi) * k + i] = dv;
        I[static_cast<size_t>(qi) * k + i] = iv;
    }
    }
}

// Device-side fallback: gather / scatter of the overflowed queries.
__global__ void fb_gather_kernel(const int32_t* __restrict__ ovf, const float* __restrict__ q,
                                 const int64_t* __restrict__ probes, int nprobe, int d, int cap, float* __restrict__ fq,
                                 int64_t* __restrict__ fprobes, int32_t* __restrict__ fcount) {
    const int cnt = min(ovf[0], cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) *fcount = cnt;
    for (int i = blockIdx.x; i < cnt; i += gridDim.x) {
        const int qi = ovf[1 + i];
        for (int j = threadIdx.x; j < d; j += blockDim.x) fq[static_cast<size_t>(i) * d + j] = q[static_cast<size_t>(qi) * d + j];
        for (int j = threadIdx.x; j < nprobe; j += blockDim.x)
            fprobes[static_cast<size_t>(i) * nprobe + j] = probes[static_cast<size_t>(qi) * nprobe + j];
    }
}

__global__ void fb_scatter_kernel(const int32_t* __restrict__ ovf, const float* __restrict__ fD,
                                  const int64_t* __restrict__ fI, int k, int cap, float* __restrict__ D,
                                  int64_t* __restrict__ I, unsigned long long* total) {
    const int cnt = min(ovf[0], cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(total, static_cast<unsigned long long>(cnt));
    for (int i = blockIdx.x; i < cnt; i += gridDim.x) {
        const int qi = ovf[1 + i];
        for (int j = threadIdx.x; j < k; j += blockDim.x) {
            D[static_cast<size_t>(qi) * k + j] = fD[static_cast<size_t>(i) * k + j];
            I[static_cast<size_t>(qi) * k + j] = fI[static_cast<size_t>(i) * k + j];
        }
    }
}

__global__ void fill_f32_kernel(float* p, int64_t n, float v) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        p[i] = v;
}

inline int grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    if (g > (1 << 30)) g = 1 << 30;
    return static_cast<int>(g < 1 ? 1 : g);
}

}  // namespace

cudaError_t launch_to_bf16_arena(const ArenaLayout& L, const float* codes, int64_t rows, void* out, cudaStream_t s) {
    const int nkb = (L.d + 63) / 64;
    cudaError_t e = cudaMemsetAsync(out, 0, bf16_image_bytes(rows, L.d), s);
    if (e != cudaSuccess) return e;
    to_bf16_arena_kernel<<<grid_for(rows * L.d, 256), 256, 0, s>>>(L, codes, rows, nkb,
                                                                    static_cast<unsigned char*>(out));
    return cudaGetLastError();
}

// Error-bound constants for dimension d (see err_coef).
// ksplit: every dimension accumulates two products (the split centroid
// image's hi and lo parts).
static void err_consts(int d, bool f8, float* cK, float* cN, bool ksplit = false) {
    const int K = (f8 ? (d + 127) / 128 * 128 : (d + 63) / 64 * 64) * (ksplit ? 2 : 1);
    const double u = 1.0 / 16777216.0, inflate = 1.0 + 1.0 / 128.0;
    *cK = static_cast<float>((K + 8) * u * inflate);
    *cN = static_cast<float>((3.0 * d + 16) * u * inflate);
}

cudaError_t launch_tighten(const float* xn, const float2* xaux, const float4* qaux, int nq, const BatchWork& w,
                           int capq, int k, int metric, int d, bool f8, int nsm, float* thr, cudaStream_t s,
                           DenseFirst df) {
    df.dense_max = std::min(df.dense_max, capq);
    float cK, cN;
    err_consts(d, f8, &cK, &cN);
    cudaError_t e = cudaMemsetAsync(w.big, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.big2, 0, sizeof(int32_t), s)) != cudaSuccess) return e;
    if (df.dense_max > 0) {
        if ((e = cudaMemsetAsync(w.rest, 0, sizeof(int32_t), s)) != cudaSuccess) return e;
        tighten_dense_kernel<<<(nq + 7) / 8, 256, 0, s>>>(xn, xaux, qaux, nq, w, capq, k, metric, cK, cN, thr, df);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    tighten_warp_kernel<<<df.dense_max > 0 ? 2 * nsm : (nq + 7) / 8, 256, 0, s>>>(xn, xaux, qaux, nq, w, capq, k,
                                                                                  metric, cK, cN, thr, df);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    tighten_warp2_kernel<<<2 * nsm, 256, 0, s>>>(xn, xaux, qaux, w, capq, k, metric, cK, cN, thr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t smem = static_cast<size_t>(capq) * 8;
    if ((e = cudaFuncSetAttribute(tighten_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem))) != cudaSuccess)
        return e;
    tighten_kernel<<<2 * nsm, 256, smem, s>>>(xn, xaux, qaux, w, capq, k, metric, cK, cN, thr);
    return cudaGetLastError();
}

cudaError_t launch_fb_gather(const int32_t* ovf, const float* q, const int64_t* probes, int nprobe, int d, int cap,
                             float* fq, int64_t* fprobes, int32_t* fcount, cudaStream_t s) {
    fb_gather_kernel<<<64, 128, 0, s>>>(ovf, q, probes, nprobe, d, cap, fq, fprobes, fcount);
    return cudaGetLastError();
}

cudaError_t launch_fb_scatter(const int32_t* ovf, const float* fD, const int64_t* fI, int k, int cap, float* D,
                              int64_t* I, unsigned long long* total, cudaStream_t s) {
    fb_scatter_kernel<<<64, 128, 0, s>>>(ovf, fD, fI, k, cap, D, I, total);
    return cudaGetLastError();
}

cudaError_t launch_centroid_image(const float* cent, int nlist, int d, void* img, float2* aux, float2* tile_aux,
                                  float* xn, cudaStream_t s) {
    const int64_t rows = (static_cast<int64_t>(nlist) + TM - 1) / TM * TM;
    const int nkb = (d + 63) / 64;  // 64-dimension blocks (two k-blocks each in the image)
    rowmajor_image_kernel<<<grid_for(rows * nkb * 64, 256), 256, 0, s>>>(cent, nlist, d, nkb, rows,
                                                                         static_cast<unsigned char*>(img));
    rowmajor_aux_kernel<<<grid_for(rows * 32, 256), 256, 0, s>>>(cent, nlist, d, rows, aux, xn);
    tile_aux_kernel<<<grid_for(rows / TM * 32, 256), 256, 0, s>>>(aux, rows / TM, tile_aux);
    return cudaGetLastError();
}

cudaError_t launch_coarse_items(int nq, int nlist, int ngroups, int nslices, int64_t* list_off, int32_t* list_size,
                                const BatchWork& w, cudaStream_t s) {
    const int64_t rows = (static_cast<int64_t>(nlist) + TM - 1) / TM * TM;
    const int64_t n = std::max<int64_t>(nq, static_cast<int64_t>(ngroups) * nslices);
    coarse_items_kernel<<<grid_for(std::max<int64_t>(n, 1), 256), 256, 0, s>>>(nq, nlist, rows, ngroups, nslices,
                                                                              list_off, list_size, w);
    return cudaGetLastError();
}

size_t coarse_refine_smem(int nlist, int d, int warps) {
    (void)nlist;
    return static_cast<size_t>(warps) * refine_warp_bytes(d);
}

cudaError_t launch_coarse_refine(float2* cand, int nq, int nlist, const float* q, const float* cent,
                                 const float* cxn, const float2* caux, const float4* qaux, int d, int metric, int m,
                                 int64_t* out_idx, float* out_score, int* err, cudaStream_t s) {
    float cK, cN;
    err_consts(d, false, &cK, &cN, true);  // the split centroid image
    int warps = 4;
    while (warps > 1 && coarse_refine_smem(nlist, d, warps) > 200 * 1024) warps >>= 1;
    const size_t smem = coarse_refine_smem(nlist, d, warps);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    const dim3 grid((nq + warps - 1) / warps);
    auto run = [&](auto kern) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * warps, smem, s>>>(cand, nq, nlist, q, cent, cxn, caux, qaux, cK, cN, d, m, out_idx,
                                            out_score, err);
        return cudaGetLastError();
    };
    if (nlist > 2048) return cudaErrorInvalidValue;
    if (metric == METRIC_L2)
        return nlist <= 1024 ? run(coarse_refine_kernel<METRIC_L2, 32>) : run(coarse_refine_kernel<METRIC_L2, 64>);
    return nlist <= 1024 ? run(coarse_refine_kernel<METRIC_IP, 32>) : run(coarse_refine_kernel<METRIC_IP, 64>);
}

cudaError_t launch_coarse_thr(const float2* cand, int nq, int S, int m, const float* cxn, const float2* caux,
                              const float4* qaux, int d, int metric, float* thr, cudaStream_t s) {
    if (S > 1024 || m > S) return cudaErrorInvalidValue;
    float cK, cN;
    err_consts(d, false, &cK, &cN, true);  // the split centroid image
    coarse_thr_kernel<<<(nq + 7) / 8, 256, 0, s>>>(cand, nq, S, m, cxn, caux, qaux, metric, cK, cN, thr);
    return cudaGetLastError();
}

cudaError_t launch_coarse_refine_keys(uint64_t* cand, const int32_t* ccnt, int nq, int stride, const float* q,
                                      const float* cent, const float* cxn, const float2* caux, const float4* qaux,
                                      int d, int metric, int m, int64_t* out_idx, float* out_score, int* err,
                                      cudaStream_t s) {
    int warps = 4;
    while (warps > 1 && coarse_refine_smem(0, d, warps) > 200 * 1024) warps >>= 1;
    const size_t smem = coarse_refine_smem(0, d, warps);
    if (smem > 200 * 1024 || m > 256) return cudaErrorInvalidValue;
    float cK, cN;
    err_consts(d, false, &cK, &cN, true);  // the split centroid image
    const dim3 grid((nq + warps - 1) / warps);
    auto run = [&](auto kern) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kern<<<grid, 32 * warps, smem, s>>>(cand, ccnt, nq, stride, q, cent, cxn, caux, qaux, d, m, cK, cN, out_idx,
                                            out_score, err);
        return cudaGetLastError();
    };
    return metric == METRIC_L2 ? run(coarse_refine_keys_kernel<METRIC_L2>) : run(coarse_refine_keys_kernel<METRIC_IP>);
}

cudaError_t launch_fill_f32(float* p, int64_t n, float v, cudaStream_t s) {
    fill_f32_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t launch_prep_queries(const float* q, int nq, int d, void* qb, float4* qaux, float* qscale, cudaStream_t s,
                                float amax, int32_t* qexact) {
    if (qscale) {
        prep_queries_f8_kernel<<<nq, 128, 0, s>>>(q, nq, d, (d + 127) / 128, static_cast<unsigned char*>(qb), qaux,
                                                  qscale);
    } else {
        if (d > PREP_DMAX) return cudaErrorInvalidValue;
        prep_queries_kernel<<<(nq + PREP_WARPS - 1) / PREP_WARPS, 32 * PREP_WARPS, 0, s>>>(
            q, nq, d, (d + 63) / 64, static_cast<__nv_bfloat16*>(qb), qaux, amax, qexact);
    }
    return cudaGetLastError();
}

cudaError_t launch_arena_integral(const float* codes, int64_t n, const float* xn, int64_t rows, int* flag,
                                  unsigned int* maxxn, cudaStream_t s) {
    arena_integral_kernel<<<1184, 256, 0, s>>>(codes, n, xn, rows, flag, maxxn);
    return cudaGetLastError();
}

cudaError_t launch_to_f8_arena(const ArenaLayout& L, const float* codes, int64_t rows, const int64_t* list_off,
                               const int32_t* list_size, int nlist, float* tile_max, float* lscale, float* tscale,
                               void* out, cudaStream_t s) {
    const int64_t tiles = rows / TM;
    cudaError_t e = cudaMemsetAsync(out, 0, f8_image_bytes(rows, L.d), s);
    if (e != cudaSuccess) return e;
    fill_f32_kernel<<<grid_for(tiles, 256), 256, 0, s>>>(tscale, tiles, 1.0f);
    tile_absmax_kernel<<<grid_for(tiles * 32, 256), 256, 0, s>>>(L, codes, tiles, tile_max);
    list_scale_kernel<<<grid_for(nlist, 128), 128, 0, s>>>(list_off, list_size, nlist, tile_max, lscale, tscale);
    to_f8_arena_kernel<<<grid_for(rows * L.d, 256), 256, 0, s>>>(L, codes, rows, (L.d + 127) / 128, tscale,
                                                                  static_cast<unsigned char*>(out));
    return cudaGetLastError();
}

cudaError_t launch_row_aux(const ArenaLayout& L, const float* codes, int64_t rows, const float* tscale, float2* aux,
                           float2* tile_aux, cudaStream_t s) {
    row_aux_kernel<<<grid_for(rows * 32, 256), 256, 0, s>>>(L, codes, rows, tscale, aux);
    const int64_t tiles = rows / TM;
    tile_aux_kernel<<<grid_for(tiles * 32, 256), 256, 0, s>>>(aux, tiles, tile_aux);
    return cudaGetLastError();
}

cudaError_t launch_tile_max(const float* xn, int64_t rows, float* tile_max, cudaStream_t s) {
    const int64_t tiles = rows / TM;
    tile_max_kernel<<<grid_for(tiles * 32, 256), 256, 0, s>>>(xn, tiles, tile_max);
    return cudaGetLastError();
}

cudaError_t launch_invert_probes(const int64_t* probes, int nq, int nprobe, int j0, int j1, int nlist,
                                 const int32_t* list_size, int rs, int qg, const BatchWork& w, cudaStream_t s) {
    const int64_t n = static_cast<int64_t>(nq) * (j1 - j0);
    cudaError_t e;
    if ((e = cudaMemsetAsync(w.pair_cnt, 0, nlist * sizeof(int32_t), s)) != cudaSuccess) return e;
    if (nlist <= INVERT_SMEM_LISTS && w.done) {
        // Up to about one CTA of 512 threads per SM (at least 1024 pairs each).
        const int64_t per = std::max<int64_t>(1024, (n + 147) / 148);
        const int nblk = static_cast<int>(std::max<int64_t>(1, (n + per - 1) / per));
        invert_count_kernel<<<nblk, 512, static_cast<size_t>(nlist) * 4, s>>>(probes, nq, nprobe, j0, j1, nlist, per,
                                                                              list_size, rs, qg, w);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const int fblk = std::max(nblk, (nlist + 15) / 16 < 148 ? (nlist + 15) / 16 : 148);
        const int64_t fper = (n + fblk - 1) / fblk;
        invert_fill_kernel<<<fblk, 512, static_cast<size_t>(nlist) * 8, s>>>(probes, nq, nprobe, j0, j1, nlist,
                                                                             std::max<int64_t>(fper, 1), list_size, rs,
                                                                             w);
        return cudaGetLastError();
    }
    if ((e = cudaMemsetAsync(w.pair_fill, 0, nlist * sizeof(int32_t), s)) != cudaSuccess) return e;
    if (nlist <= INVERT_SMEM_LISTS) {
        // About 160 CTAs of 512 threads (at least 512 pairs each).
        const int64_t per = std::max<int64_t>(512, (n + 159) / 160);
        const int nblk = static_cast<int>(std::max<int64_t>(1, (n + per - 1) / per));
        probe_hist_smem_kernel<<<nblk, 512, static_cast<size_t>(nlist) * 4, s>>>(probes, nq, nprobe, j0, j1, nlist,
                                                                                 per, w.pair_cnt);
        scan_kernel<<<1, 1024, 0, s>>>(w.pair_cnt, nlist, w.pair_off);
        probe_fill_smem_kernel<<<nblk, 512, static_cast<size_t>(nlist) * 8, s>>>(probes, nq, nprobe, j0, j1, nlist,
                                                                                 per, w.pair_off, w.pair_fill, w.pairs);
    } else {
        probe_hist_kernel<<<grid_for(n, 256), 256, 0, s>>>(probes, nq, nprobe, j0, j1, w.pair_cnt);
        scan_kernel<<<1, 1024, 0, s>>>(w.pair_cnt, nlist, w.pair_off);
        probe_fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(probes, nq, nprobe, j0, j1, w.pair_off, w.pair_fill,
                                                           w.pairs);
    }
    item_count_kernel<<<grid_for(nlist, 256), 256, 0, s>>>(w.pair_cnt, list_size, nlist, rs, qg, w.item_cnt);
    scan_kernel<<<1, 1024, 0, s>>>(w.item_cnt, nlist, w.item_off);
    item_fill_kernel<<<grid_for(static_cast<int64_t>(nlist) * 32, 256), 256, 0, s>>>(w.item_off, list_size, nlist, rs,
                                                                                     w.item_cap, w.items);
    return cudaGetLastError();
}

int batched_group_size(int d, bool f8) {
    const int nkb = f8 ? (d + 127) / 128 : (d + 63) / 64;
    if (batched_stages<128>(nkb)) return 128;
    if (batched_stages<64>(nkb)) return 64;
    if (batched_stages<32>(nkb)) return 32;
    return 0;
}

template <int QG, bool F8>
static cudaError_t launch_batched_t(BatchedParams p, int nsm, cudaStream_t s) {
    p.nslot = SLOT_MAX;
    p.ns = batched_stages<QG>(p.nkb >> p.ksplit, SLOT_MAX);
    if (p.ns < NS_SLOT3) {
        p.nslot = 2;
        p.ns = batched_stages<QG>(p.nkb >> p.ksplit, 2);
    }
    if (p.ns == 0) return cudaErrorInvalidValue;
    const size_t smem = batched_smem<QG>(p.nkb >> p.ksplit, p.ns, p.nslot);
    cudaError_t e = cudaFuncSetAttribute(batched_scan_kernel<QG, F8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    batched_scan_kernel<QG, F8><<<nsm, BATCH_THREADS, smem, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_batched_scan(const BatchedLaunch& b, const BatchWork& w, int* err, cudaStream_t s) {
    BatchedParams p;
    p.abf = static_cast<const unsigned char*>(b.abf);
    p.list_off = b.list_off;
    p.list_size = b.list_size;
    p.item_off = w.item_off;
    p.items = w.items;
    p.item_cap = w.item_cap;
    p.pair_off = w.pair_off;
    p.pairs = w.pairs;
    p.pair_cnt = w.pair_cnt;
    p.xn = b.xn;
    p.tile_aux = b.tile_aux;
    p.qb = static_cast<const unsigned char*>(b.qb);
    p.qaux = b.qaux;
    p.lscale = b.lscale;
    p.qscale = b.qscale;
    p.thr = b.thr;
    p.cand = w.cand;
    p.cand_cnt = w.cand_cnt;
    p.work = w.work;
    p.err = err;
    p.nlist = b.nlist;
    p.ksplit = b.ksplit ? 1 : 0;
    p.nkb = (b.f8 ? (b.d + 127) / 128 : (b.d + 63) / 64) << p.ksplit;
    p.rs = b.rs;
    p.capq = b.capq;
    p.metric = b.metric;
    p.dense_max = std::min(b.dense_max, b.capq);
    p.xaux = b.xaux;
    err_consts(b.d, b.f8, &p.cK, &p.cN, b.ksplit);
    cudaError_t e;
    if ((e = cudaMemsetAsync(w.work, 0, sizeof(unsigned int), s)) != cudaSuccess) return e;
    switch (b.qg * 2 + (b.f8 ? 1 : 0)) {
        case 256: return launch_batched_t<128, false>(p, b.nsm, s);
        case 257: return launch_batched_t<128, true>(p, b.nsm, s);
        case 128: return launch_batched_t<64, false>(p, b.nsm, s);
        case 129: return launch_batched_t<64, true>(p, b.nsm, s);
        case 64: return launch_batched_t<32, false>(p, b.nsm, s);
        case 65: return launch_batched_t<32, true>(p, b.nsm, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_rerank(const ArenaLayout& L, const float* codes, const int64_t* ids, const float* xn,
                          const float2* xaux, const float4* qaux, const float* q, int nq, const BatchWork& w, int qbase,
                          int capq, int k, int rmax, int metric, bool f8, int nsm, float* D, int64_t* I,
                          cudaStream_t s, const int32_t* qexact) {
    float cK, cN;
    err_consts(L.d, f8, &cK, &cN);
    cudaError_t e = cudaMemsetAsync(w.big, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    const size_t wsmem = static_cast<size_t>(8) * (256 * sizeof(uint64_t) + L.row_pitch * sizeof(float));
    if ((e = cudaFuncSetAttribute(rerank_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(wsmem))) != cudaSuccess)
        return e;
    rerank_warp_kernel<<<(nq + 7) / 8, 256, wsmem, s>>>(L, codes, ids, xn, xaux, qaux, q, nq, w, capq, k, rmax, metric,
                                                        cK, cN, qexact, D, I);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t smem = static_cast<size_t>(RERANK_MAX) * 8 + static_cast<size_t>(L.row_pitch) * 4 +
                        static_cast<size_t>(capq) * 8;
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    if ((e = cudaFuncSetAttribute(rerank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem))) != cudaSuccess)
        return e;
    rerank_kernel<<<2 * nsm, 256, smem, s>>>(L, codes, ids, xn, xaux, qaux, q, w, qbase, capq, k, rmax, metric, cK, cN,
                                             qexact, D, I);
    return cudaGetLastError();
}

}  // namespace hy
