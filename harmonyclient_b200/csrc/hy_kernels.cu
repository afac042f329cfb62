// IVF kernels for B200 (sm_100a): coarse quantisation, selection, warm-up
// thresholds, the plain FP32 list scan with dimension-block pruning, the final
// top-k merge, and the index-construction kernels (k-means, add).
//
// Arithmetic note: every distance is accumulated dimension by dimension in
// increasing order with separately rounded multiply and add (__fmul_rn /
// __fadd_rn, no FMA contraction), so each float result is bit-identical to the
// project's sequential CPU restatement of the reference (the oracle).  The
// plain scan accumulates each dimension block from zero and adds the block
// sums in order, which is the order of the reference's 4-chunk pruning loop
// (src/node.cpp:640-656).
#include <algorithm>
#include <cfloat>
#include <cub/device/device_radix_sort.cuh>

#include "hy_common.cuh"
#include "hy_kernels.cuh"

namespace hy {

namespace {

constexpr int METRIC_IP = 0;
constexpr int METRIC_L2 = 1;

// ---------------------------------------------------------------------------
// Coarse scores: out[i][c] = ||q_i - c||^2 (L2) or -<q_i, c> (IP), so that
// smaller is better for both metrics.  64 queries x 64 centroids per CTA,
// 4 x 4 outputs per thread, dimensions staged 32 at a time in shared memory.
// (The reference computes these with IVFScan::lite_scan_codes over all
// centroids, src/IVFScan.hpp:108-138, src/Index.cpp:985-990.)
template <int METRIC>
__global__ void __launch_bounds__(256) coarse_scores_kernel(const float* __restrict__ q, int nq,
                                                            const float* __restrict__ c, int nlist, int d,
                                                            float* __restrict__ out) {
    __shared__ __align__(16) float Qs[32][68];
    __shared__ __align__(16) float Cs[32][68];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int q0 = blockIdx.y * 64, c0 = blockIdx.x * 64;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;

    for (int d0 = 0; d0 < d; d0 += 32) {
        for (int i = threadIdx.x; i < 64 * 32; i += 256) {
            const int r = i >> 5, j = i & 31;
            const int gj = d0 + j;
            const int gq = q0 + r, gc = c0 + r;
            Qs[j][r] = (gq < nq && gj < d) ? q[static_cast<size_t>(gq) * d + gj] : 0.0f;
            Cs[j][r] = (gc < nlist && gj < d) ? c[static_cast<size_t>(gc) * d + gj] : 0.0f;
        }
        __syncthreads();
        const int jn = min(32, d - d0);
        for (int j = 0; j < jn; ++j) {
            const float4 a = *reinterpret_cast<const float4*>(&Qs[j][ty * 4]);
            const float4 b = *reinterpret_cast<const float4*>(&Cs[j][tx * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w};
            const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    acc[u][v] = METRIC == METRIC_L2 ? sq_add(acc[u][v], av[u], bv[v]) : ip_add(acc[u][v], av[u], bv[v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int gq = q0 + ty * 4 + u;
        if (gq >= nq) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int gc = c0 + tx * 4 + v;
            if (gc < nlist) out[static_cast<size_t>(gq) * nlist + gc] = METRIC == METRIC_L2 ? acc[u][v] : -acc[u][v];
        }
    }
}

// Per row of `scores` (n values, smaller is better): the m best, best first,
// ties broken by lower column.  One CTA per row.
__global__ void __launch_bounds__(256) select_kernel(const float* __restrict__ scores, int n, int m,
                                                     int64_t* __restrict__ out_idx, float* __restrict__ out_score) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int P = next_pow2(m);
    uint64_t* sel = reinterpret_cast<uint64_t*>(sm);
    uint32_t* vals = reinterpret_cast<uint32_t*>(sel + P);
    __shared__ int hist[256];
    __shared__ uint32_t sh[2];
    __shared__ int scratch[34];
    const size_t row = blockIdx.x;
    const float* src = scores + row * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) vals[i] = f2o(src[i]);
    for (int i = threadIdx.x; i < P; i += blockDim.x) sel[i] = KEY_MAX;
    __syncthreads();
    int need;
    const uint32_t vstar = cta_radix_select(vals, n, m, &need, hist, sh);
    cta_collect(vals, n, m, vstar, need, sel, scratch);
    cta_bitonic_sort(sel, P);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const uint64_t key = sel[i];
        out_idx[row * m + i] = static_cast<int64_t>(key & 0xffffffffu);
        if (out_score) out_score[row * m + i] = o2f(static_cast<uint32_t>(key >> 32));
    }
}

// Warp version of select_kernel (one warp per row) for rows of at most
// 32*SPER values and m <= 256: the m-th smallest ordered key by a warp radix
// select, every smaller element plus the lowest-column equal ones collected
// through a per-warp shared list, then a register bitonic sort.  Same result
// as select_kernel.
template <int SPER>
__global__ void __launch_bounds__(256) select_warp_kernel(const float* __restrict__ scores, int nrows, int n, int m,
                                                          int64_t* __restrict__ out_idx,
                                                          float* __restrict__ out_score) {
    __shared__ int hist[8][256];
    __shared__ uint64_t list[8][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row = static_cast<int64_t>(blockIdx.x) * 8 + warp;
    if (row >= nrows) return;  // whole warp
    const float* src = scores + row * n;
    uint32_t v[SPER];
#pragma unroll
    for (int r = 0; r < SPER; ++r) {
        const int e = r * 32 + lane;
        v[r] = e < n ? f2o(src[e]) : 0xffffffffu;
    }
    const uint32_t vstar = warp_radix_select<SPER>(v, n, m, hist[warp], lane);
    int less = 0;
#pragma unroll
    for (int r = 0; r < SPER; ++r) less += (r * 32 + lane < n && v[r] < vstar) ? 1 : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) less += __shfl_xor_sync(FULL, less, o);
    int need = m - less;  // equal elements to take, lowest columns first
    int pos = 0;
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < SPER; ++r) {
        const int e = r * 32 + lane;
        const bool lt = e < n && v[r] < vstar;
        const bool eq = e < n && v[r] == vstar;
        const unsigned be = __ballot_sync(FULL, eq);
        const bool take = lt || (eq && __popc(be & below) < need);
        need -= min(__popc(be), max(need, 0));
        const unsigned bt = __ballot_sync(FULL, take);
        if (take) list[warp][pos + __popc(bt & below)] = (static_cast<uint64_t>(v[r]) << 32) | static_cast<uint32_t>(e);
        pos += __popc(bt);
    }
    __syncwarp();
    uint64_t kk[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int e = r * 32 + lane;
        kk[r] = e < m ? list[warp][e] : KEY_MAX;
    }
    warp_sort<8>(kk, lane);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int e = r * 32 + lane;
        if (e < m) {
            out_idx[row * m + e] = static_cast<int64_t>(kk[r] & 0xffffffffu);
            if (out_score) out_score[row * m + e] = o2f(static_cast<uint32_t>(kk[r] >> 32));
        }
    }
}

// Per row: the first minimum (lowest column among equal minima), one warp per
// row — the reference's nearest-centroid rule (strict < in column order,
// src/IVFScan.hpp:131, src/Clustering.cpp:107).
__global__ void argmin_kernel(const float* __restrict__ scores, int nrows, int n, int64_t* __restrict__ out_idx,
                              float* __restrict__ out_score) {
    const int lane = threadIdx.x & 31;
    const int64_t row = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (row >= nrows) return;
    const float* src = scores + row * n;
    float best = INFINITY;
    int bi = n;
    for (int i = lane; i < n; i += 32) {
        const float v = src[i];
        if (v < best) {
            best = v;
            bi = i;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(FULL, best, o);
        const int oi = __shfl_xor_sync(FULL, bi, o);
        if (ob < best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    if (lane == 0) {
        out_idx[row] = bi < n ? bi : 0;
        if (out_score) out_score[row] = best;
    }
}

// Warm-up thresholds (Index::warmUpSearch, src/Index.cpp:999-1051, and the
// heapTops read at src/Index.cpp:1300-1303): per query, the k-th smallest L2
// distance over the first min(wls, |l|) rows of its first min(wl, nprobe)
// probed lists; FLT_MAX when fewer than k rows were seen.  One CTA per query;
// distances are collected in shared memory and the k-th found by radix
// selection.
// True when query qi's nearest list has between skip_lo and skip_hi rows.
__device__ inline bool warmup_skipped(const int32_t* list_size, const int64_t* probes, int qi, int nprobe, int skip_lo,
                                      int skip_hi) {
    if (skip_hi < skip_lo) return false;
    const int64_t l0 = probes[static_cast<size_t>(qi) * nprobe];
    if (l0 < 0) return false;
    const int sz = list_size[l0];
    return sz >= skip_lo && sz <= skip_hi;
}

__global__ void __launch_bounds__(256) warmup_kernel(ArenaLayout L, const float* __restrict__ codes,
                                                     const int64_t* __restrict__ list_off,
                                                     const int32_t* __restrict__ list_size,
                                                     const float* __restrict__ q, const int64_t* __restrict__ probes,
                                                     int nprobe, int k, int wl, int wls, int blockwise,
                                                     uint32_t* __restrict__ out_thr, float* __restrict__ out_f,
                                                     int skip_lo, int skip_hi) {
    extern __shared__ __align__(16) unsigned char sm[];
    float* qs = reinterpret_cast<float*>(sm);
    int* rbase = reinterpret_cast<int*>(qs + L.row_pitch);  // [wl+1] prefix of rows
    int64_t* r0 = reinterpret_cast<int64_t*>(rbase + ((wl + 2) & ~1));
    uint32_t* vals = reinterpret_cast<uint32_t*>(r0 + wl);
    __shared__ int hist[256];
    __shared__ uint32_t sh[2];
    const int qi = blockIdx.x;
    const int wle = min(wl, nprobe);
    if (warmup_skipped(list_size, probes, qi, nprobe, skip_lo, skip_hi)) {
        if (threadIdx.x == 0) {
            out_thr[qi] = f2o(FLT_MAX);
            if (out_f) out_f[qi] = FLT_MAX;
        }
        return;  // whole block
    }
    stage_query(L, q + static_cast<size_t>(qi) * L.d, qs);
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int j = 0; j < wle; ++j) {
            const int64_t l = probes[static_cast<size_t>(qi) * nprobe + j];
            rbase[j] = acc;
            r0[j] = l >= 0 ? list_off[l] : 0;
            acc += l >= 0 ? min(wls, static_cast<int>(list_size[l])) : 0;
        }
        rbase[wle] = acc;
    }
    __syncthreads();
    const int total = rbase[wle];
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int j = 0;
        while (rbase[j + 1] <= i) ++j;
        const int64_t r = r0[j] + (i - rbase[j]);
        vals[i] = f2o(row_l2_global(L, codes, r, qs, blockwise != 0));
    }
    __syncthreads();
    float thr = FLT_MAX;
    if (total >= k) {
        int need;
        const uint32_t v = cta_radix_select(vals, total, k, &need, hist, sh);
        thr = o2f(v);
    }
    if (threadIdx.x == 0) {
        out_thr[qi] = f2o(thr);
        if (out_f) out_f[qi] = thr;
    }
}

// Warp version of warmup_kernel (one warp per query) for at most 32 warm-up
// lists and 1024 warm-up rows: the same distances (row_l2_global), the k-th
// by a warp radix select.
__global__ void __launch_bounds__(256) warmup_warp_kernel(const __grid_constant__ ArenaLayout L,
                                                          const float* __restrict__ codes,
                                                          const int64_t* __restrict__ list_off,
                                                          const int32_t* __restrict__ list_size,
                                                          const float* __restrict__ q,
                                                          const int64_t* __restrict__ probes, int nq, int nprobe,
                                                          int k, int wl, int wls, int blockwise,
                                                          uint32_t* __restrict__ out_thr, float* __restrict__ out_f,
                                                          int skip_lo, int skip_hi) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ int hist[8][256];
    __shared__ int s_base[8][33];
    __shared__ int64_t s_r0[8][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * 8 + warp;
    if (qi >= nq) return;  // whole warp
    if (warmup_skipped(list_size, probes, qi, nprobe, skip_lo, skip_hi)) {
        if (lane == 0) {
            out_thr[qi] = f2o(FLT_MAX);
            if (out_f) out_f[qi] = FLT_MAX;
        }
        return;  // whole warp
    }
    float* qs = reinterpret_cast<float*>(sm) + static_cast<size_t>(warp) * L.row_pitch;
    const float* src = q + static_cast<size_t>(qi) * L.d;
    for (int i = lane; i < L.row_pitch; i += 32) {
        int b = 0;
        while (b + 1 < L.nb && i >= L.boff[b + 1]) ++b;
        const int j = i - L.boff[b];
        qs[i] = j < L.bstart[b + 1] - L.bstart[b] ? src[L.bstart[b] + j] : 0.0f;
    }
    const int wle = min(wl, nprobe);
    int cnt = 0;
    int64_t r0 = 0;
    if (lane < wle) {
        const int64_t l = probes[static_cast<size_t>(qi) * nprobe + lane];
        if (l >= 0) {
            cnt = min(wls, static_cast<int>(list_size[l]));
            r0 = list_off[l];
        }
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    s_base[warp][lane] = incl - cnt;
    s_r0[warp][lane] = r0;
    const int total = __shfl_sync(FULL, incl, 31);
    if (lane == 0) s_base[warp][32] = total;
    __syncwarp();
    uint32_t v[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        const int i = r * 32 + lane;
        v[r] = 0xffffffffu;
        if (i < total) {
            int j = 0;
            while (s_base[warp][j + 1] <= i) ++j;
            const int64_t row = s_r0[warp][j] + (i - s_base[warp][j]);
            v[r] = f2o(row_l2_global(L, codes, row, qs, blockwise != 0));
        }
    }
    float thr = FLT_MAX;
    if (total >= k) thr = o2f(warp_radix_select<32>(v, total, k, hist[warp], lane));
    if (lane == 0) {
        out_thr[qi] = f2o(thr);
        if (out_f) out_f[qi] = thr;
    }
}

// ---------------------------------------------------------------------------
// The plain FP32 list scan.
//
// Grid: one CTA per (query, split); split s handles probes j = s, s+nsplit, ...
// (the reference's vector partition across teams becomes a partition of the
// probe list across CTAs).  Each CTA enumerates the 32-row tiles of its lists
// and its warps take tiles from a shared counter.  A warp runs S independent
// tile slots: each slot loads one dimension block of its tile with a bulk
// copy, accumulates the block into every lane's partial distance (lane = row),
// prunes rows whose partial exceeds the query's running threshold, and loads
// the next block only if some row of the tile is still alive — so pruned
// tiles stop costing HBM bytes (the reference's DIVIDE_DIM / in-rank 4-chunk
// prune, src/node.cpp:634-657 and 1055-1114, moved inside one kernel).
// Survivors enter a per-warp candidate buffer.  The CTA keeps one sorted
// top-K' (K' = 32*KR >= k) in shared memory; a warp whose buffer fills takes
// the CTA's merge lock, merges its candidates into that list with register
// bitonic networks and lowers the CTA threshold to the list's k-th key, so
// the threshold reflects every row the CTA has seen.  At the end the list
// holds the CTA's K' best keys.
//
// Threshold = min(warm-up threshold, the CTA list's k-th key, the k-th key
// published by other splits of the query).  Each is an upper bound
// on the query's final k-th distance, so pruning (partial > threshold) and
// admission (distance <= threshold) never drop a row of the exact top-k.
template <int KR, int S>
__global__ void __launch_bounds__(512, 1) scan_plain_kernel(const __grid_constant__ ScanParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int KP = KR * 32;
    constexpr int CAP = 2 * KP;
    const ArenaLayout& L = p.L;
    const int W = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int split = blockIdx.x % p.nsplit;
    // Queries of this CTA: blockIdx.x / nsplit, then every (grid / nsplit)-th
    // after it, below the device count when one is given (a grid of nq *
    // nsplit CTAs takes one query each).
    const int nq_eff = p.nq_dev ? min(*p.nq_dev, p.nq) : p.nq;
    const int qstride = gridDim.x / p.nsplit;
    if (static_cast<int>(blockIdx.x / p.nsplit) >= nq_eff) return;  // whole CTA, before any barrier
    const int npc = (p.nprobe - split + p.nsplit - 1) / p.nsplit;  // probes of this CTA
    const int npa = ((p.nprobe + p.nsplit - 1) / p.nsplit + 3) & ~3;  // table entries, padded for alignment
    const size_t slot_floats = static_cast<size_t>(32) * L.max_pitch;

    float* bufs = reinterpret_cast<float*>(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(bufs + static_cast<size_t>(W) * S * slot_floats);
    uint64_t* cand = bars + W * S;
    uint64_t* ctop = cand + W * CAP;  // the CTA's sorted top-K'
    int64_t* s_row0 = reinterpret_cast<int64_t*>(ctop + KP);
    float* qs = reinterpret_cast<float*>(s_row0 + npa);
    int* s_size = reinterpret_cast<int*>(qs + L.row_pitch);
    int* s_pref = s_size + npa;
    __shared__ unsigned int s_thr;
    __shared__ int s_next, s_ntiles, s_lock;

    if (threadIdx.x == 0) {
        for (int i = 0; i < W * S; ++i) mbar_init(&bars[i], 1);
        fence_mbar_init();
    }
    // Barrier phases carry over from one query to the next: every copy a
    // query issues is waited for before its scan ends.
    uint32_t sphase[S];
#pragma unroll
    for (int s = 0; s < S; ++s) sphase[s] = 0;

    for (int qi = blockIdx.x / p.nsplit; qi < nq_eff; qi += qstride) {
    // The previous query's result has been copied out (and, first time, the
    // barriers are initialised) before the shared state is set up again.
    __syncthreads();
    // --- CTA setup: query, probe table (tile prefix), threshold.
    stage_query(L, p.q + static_cast<size_t>(qi) * L.d, qs);
    if (warp == 0) {
        int carry = 0;
        for (int base = 0; base < npc; base += 32) {
            const int m = base + lane;
            int tiles = 0;
            if (m < npc) {
                const int64_t l = p.probes[static_cast<size_t>(qi) * p.nprobe + split + static_cast<size_t>(m) * p.nsplit];
                int sz = 0;
                int64_t r0 = 0;
                if (l >= 0) {
                    sz = p.list_size[l];
                    r0 = p.list_off[l];
                }
                s_size[m] = sz;
                s_row0[m] = r0;
                tiles = (sz + 31) >> 5;
            }
            int incl = tiles;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += t;
            }
            if (m < npc) s_pref[m] = carry + incl;
            carry += __shfl_sync(FULL, incl, 31);
        }
        if (lane == 0) {
            s_ntiles = carry;
            s_next = 0;
            s_lock = 0;
            s_thr = p.init_thr ? p.init_thr[qi] : 0xffffffffu;
        }
    }
    for (int i = threadIdx.x; i < KP; i += blockDim.x) ctop[i] = KEY_MAX;
    __syncthreads();

    const int ntiles = s_ntiles;
    float* wb = bufs + static_cast<size_t>(warp) * S * slot_floats;
    uint64_t* wbar = bars + warp * S;
    uint64_t* wc = cand + warp * CAP;
    const bool l2 = p.metric == METRIC_L2;
    const bool prune = p.prune && l2;

    int ccount = 0;
    unsigned long long loaded = 0, possible = 0;
    uint32_t gcache = p.g_thr ? p.g_thr[qi] : 0xffffffffu;

    int64_t srow[S];
    int sblk[S];
    float spart[S];
    bool salive[S];
    bool sact[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        srow[s] = 0;
        sblk[s] = 0;
        spart[s] = 0.0f;
        salive[s] = false;
        sact[s] = false;
    }

    auto read_thr = [&]() -> float {
        const uint32_t a = *reinterpret_cast<volatile unsigned int*>(&s_thr);
        const uint32_t key = a < gcache ? a : gcache;
        return key == 0xffffffffu ? INFINITY : o2f(key);
    };

    auto issue = [&](int s) {
        const int b = sblk[s];
        const uint32_t bytes = static_cast<uint32_t>(32 * L.pitch[b] * sizeof(float));
        const float* src = p.codes + static_cast<size_t>(srow[s] >> 5) * 32 * L.row_pitch + static_cast<size_t>(L.boff[b]) * 32;
        if (lane == 0) {
            fence_proxy_async();
            mbar_expect_tx(&wbar[s], bytes);
            bulk_g2s(wb + static_cast<size_t>(s) * slot_floats, src, bytes, &wbar[s]);
        }
        ++loaded;
    };

    auto grab = [&](int s) -> bool {
        int g = 0;
        if (lane == 0) g = atomicAdd(&s_next, 1);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ntiles) return false;
        int lo = 0, hi = npc - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s_pref[mid] > g)
                hi = mid;
            else
                lo = mid + 1;
        }
        const int tprev = lo ? s_pref[lo - 1] : 0;
        const int tt = g - tprev;
        srow[s] = s_row0[lo] + 32 * static_cast<int64_t>(tt);
        const int nvalid = min(32, s_size[lo] - 32 * tt);
        sblk[s] = 0;
        spart[s] = 0.0f;
        salive[s] = lane < nvalid;
        possible += L.nb;
        if (p.g_thr) gcache = *reinterpret_cast<volatile unsigned int*>(&p.g_thr[qi]);
        issue(s);
        return true;
    };

    // Merge this warp's candidates into the CTA list under the merge lock
    // (bounded spin; on timeout the device status word is raised).
    auto flush = [&]() {
        __syncwarp();
        int got = 0;
        if (lane == 0) {
            for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
                if (atomicCAS(&s_lock, 0, 1) == 0) {
                    got = 1;
                    break;
                }
                __nanosleep(32);
            }
            if (!got) atomicCAS(p.err, 0, DEV_ERR_TIMEOUT);
        }
        got = __shfl_sync(FULL, got, 0);
        if (got) {
            __threadfence_block();
            volatile uint64_t* vt = ctop;
            uint64_t t[KR];
#pragma unroll
            for (int r = 0; r < KR; ++r) t[r] = vt[r * 32 + lane];
            for (int base = 0; base < ccount; base += KP) {
                uint64_t c[KR];
#pragma unroll
                for (int r = 0; r < KR; ++r) {
                    const int idx = base + r * 32 + lane;
                    c[r] = idx < ccount ? wc[idx] : KEY_MAX;
                }
                warp_sort<KR>(c, lane);
                warp_merge<KR>(t, c, lane);
            }
#pragma unroll
            for (int r = 0; r < KR; ++r) vt[r * 32 + lane] = t[r];
            const uint64_t kth = warp_get<KR>(t, p.k - 1);
            if (kth != KEY_MAX && lane == 0) {
                const uint32_t key = static_cast<uint32_t>(kth >> 32);
                atomicMin(&s_thr, key);
                if (p.g_thr) atomicMin(&p.g_thr[qi], key);
            }
            __threadfence_block();
            __syncwarp();
            if (lane == 0) atomicExch(&s_lock, 0);
        }
        __syncwarp();
        ccount = 0;
    };

#pragma unroll
    for (int s = 0; s < S; ++s) sact[s] = grab(s);

    // Accumulate the staged block of slot s into one partial sum per lane
    // (lane = row), dimension by dimension.
    auto block_sum = [&](int s) -> float {
        const int b = sblk[s];
        const int P = L.pitch[b];
        const float* rowp = wb + static_cast<size_t>(s) * slot_floats + lane * P;
        const float* qb = qs + L.boff[b];
        float acc = 0.0f;
        for (int c8 = 0; c8 < (P >> 2); c8 += 8) {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const float4 x = *reinterpret_cast<const float4*>(rowp + 4 * (c8 + (u ^ (lane & 7))));
                const float4 y = *reinterpret_cast<const float4*>(qb + 4 * (c8 + u));
                if (l2) {
                    acc = sq_add(acc, y.x, x.x);
                    acc = sq_add(acc, y.y, x.y);
                    acc = sq_add(acc, y.z, x.z);
                    acc = sq_add(acc, y.w, x.w);
                } else {
                    acc = ip_add(acc, y.x, x.x);
                    acc = ip_add(acc, y.y, x.y);
                    acc = ip_add(acc, y.z, x.z);
                    acc = ip_add(acc, y.w, x.w);
                }
            }
        }
        return acc;
    };

    // The same for two slots whose blocks have equal pitch, interleaved so
    // the two dependent add chains overlap.
    auto block_sum2 = [&](int s0, int s1, float& a0, float& a1) {
        const int b0 = sblk[s0], b1 = sblk[s1];
        const int P = L.pitch[b0];
        const float* r0 = wb + static_cast<size_t>(s0) * slot_floats + lane * P;
        const float* r1 = wb + static_cast<size_t>(s1) * slot_floats + lane * P;
        const float* q0 = qs + L.boff[b0];
        const float* q1 = qs + L.boff[b1];
        float acc0 = 0.0f, acc1 = 0.0f;
        for (int c8 = 0; c8 < (P >> 2); c8 += 8) {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int pc = 4 * (c8 + (u ^ (lane & 7)));
                const float4 x0 = *reinterpret_cast<const float4*>(r0 + pc);
                const float4 x1 = *reinterpret_cast<const float4*>(r1 + pc);
                const float4 y0 = *reinterpret_cast<const float4*>(q0 + 4 * (c8 + u));
                const float4 y1 = *reinterpret_cast<const float4*>(q1 + 4 * (c8 + u));
                if (l2) {
                    acc0 = sq_add(acc0, y0.x, x0.x);
                    acc1 = sq_add(acc1, y1.x, x1.x);
                    acc0 = sq_add(acc0, y0.y, x0.y);
                    acc1 = sq_add(acc1, y1.y, x1.y);
                    acc0 = sq_add(acc0, y0.z, x0.z);
                    acc1 = sq_add(acc1, y1.z, x1.z);
                    acc0 = sq_add(acc0, y0.w, x0.w);
                    acc1 = sq_add(acc1, y1.w, x1.w);
                } else {
                    acc0 = ip_add(acc0, y0.x, x0.x);
                    acc1 = ip_add(acc1, y1.x, x1.x);
                    acc0 = ip_add(acc0, y0.y, x0.y);
                    acc1 = ip_add(acc1, y1.y, x1.y);
                    acc0 = ip_add(acc0, y0.z, x0.z);
                    acc1 = ip_add(acc1, y1.z, x1.z);
                    acc0 = ip_add(acc0, y0.w, x0.w);
                    acc1 = ip_add(acc1, y1.w, x1.w);
                }
            }
        }
        a0 = acc0;
        a1 = acc1;
    };

    // After slot s's block is summed: prune and continue the tile, or emit
    // candidates and take the next tile.
    auto post = [&](int s, float acc) {
        const int b = sblk[s];
        spart[s] = b == 0 ? acc : __fadd_rn(spart[s], acc);
        const float thr = read_thr();
        if (b + 1 < L.nb) {
            if (prune) salive[s] = salive[s] && !(spart[s] > thr);
            if (__any_sync(FULL, salive[s])) {
                sblk[s] = b + 1;
                issue(s);
                return;
            }
        } else {
            const float score = l2 ? spart[s] : -spart[s];
            const bool isc = salive[s] && score <= thr;
            const unsigned bal = __ballot_sync(FULL, isc);
            if (bal) {
                const int nc = __popc(bal);
                // Merge once 32 candidates are buffered (or the buffer would
                // overflow), so the CTA threshold follows the scan closely.
                if (ccount + nc > CAP || ccount >= 32) flush();
                if (isc) {
                    const int pos = ccount + __popc(bal & ((1u << lane) - 1u));
                    wc[pos] = (static_cast<uint64_t>(f2o(score)) << 32) | static_cast<uint32_t>(srow[s] + lane);
                }
                ccount += nc;
            }
        }
        sact[s] = grab(s);
    };

    for (;;) {
        bool any = false;
#pragma unroll
        for (int s0 = 0; s0 < S; s0 += 2) {
            const int s1 = s0 + 1;
            bool ok0 = sact[s0], ok1 = sact[s1];
            if (!(ok0 || ok1)) continue;
            any = true;
            if (ok0 && !mbar_wait_bounded(&wbar[s0], sphase[s0], p.err)) {
                sact[s0] = false;
                ok0 = false;
            }
            if (ok1 && !mbar_wait_bounded(&wbar[s1], sphase[s1], p.err)) {
                sact[s1] = false;
                ok1 = false;
            }
            float a0 = 0.0f, a1 = 0.0f;
            if (ok0 && ok1 && L.pitch[sblk[s0]] == L.pitch[sblk[s1]]) {
                block_sum2(s0, s1, a0, a1);
            } else {
                if (ok0) a0 = block_sum(s0);
                if (ok1) a1 = block_sum(s1);
            }
            __syncwarp();
            if (ok0) {
                sphase[s0] ^= 1u;
                post(s0, a0);
            }
            if (ok1) {
                sphase[s1] ^= 1u;
                post(s1, a1);
            }
        }
        if (!any) break;
    }
    if (ccount > 0) flush();
    if (lane == 0 && p.counters) {
        atomicAdd(&p.counters[0], loaded);
        atomicAdd(&p.counters[1], possible);
    }
    __syncthreads();
    uint64_t* dst = p.out + (static_cast<size_t>(qi) * p.nsplit + split) * KP;
    for (int i = threadIdx.x; i < KP; i += blockDim.x) dst[i] = ctop[i];
    }  // queries of this CTA
}

// Final merge: per query, the k best of nparts sorted lists of kp keys, then
// keys -> (distance, id).  Unfilled entries get the reference's heap_init
// values (FLT_MAX / -FLT_MAX, id -1; src/heap.hpp:13-25).
__global__ void __launch_bounds__(256) merge_kernel(const uint64_t* __restrict__ parts, int nq, int nparts, int kp, int k,
                                                    int metric, const int64_t* __restrict__ ids,
                                                    float* __restrict__ D, int64_t* __restrict__ I,
                                                    int64_t* __restrict__ rows, const int32_t* __restrict__ nq_dev) {
    extern __shared__ __align__(16) unsigned char sm[];
    uint64_t* a = reinterpret_cast<uint64_t*>(sm);
    // Query blockIdx.x, then every gridDim.x-th after it, below the device
    // count when one is given.
    const int nq_eff = nq_dev ? min(*nq_dev, nq) : nq;
    for (size_t qi = blockIdx.x; qi < static_cast<size_t>(nq_eff); qi += gridDim.x) {
    const int n = nparts * kp;
    const uint64_t* src = parts + qi * n;
    const uint64_t* best = src;
    if (nparts > 1) {
        const int P = next_pow2(n);
        __syncthreads();  // the previous query's keys have been read
        for (int i = threadIdx.x; i < P; i += blockDim.x) a[i] = i < n ? src[i] : KEY_MAX;
        __syncthreads();
        cta_bitonic_sort(a, P);
        best = a;
    }
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const uint64_t key = i < n ? best[i] : KEY_MAX;
        float dv;
        int64_t iv;
        if (key == KEY_MAX) {
            dv = metric == METRIC_L2 ? FLT_MAX : -FLT_MAX;
            iv = -1;
        } else {
            const float sc = o2f(static_cast<uint32_t>(key >> 32));
            dv = metric == METRIC_L2 ? sc : -sc;
            iv = ids[key & 0xffffffffu];
        }
        D[qi * k + i] = dv;
        I[qi * k + i] = iv;
        if (rows) rows[qi * k + i] = key == KEY_MAX ? -1 : static_cast<int64_t>(key & 0xffffffffu);
    }
    }  // queries of this CTA
}

// ---------------------------------------------------------------------------
// Index construction kernels.
__global__ void histogram_kernel(const int64_t* __restrict__ labels, int64_t n, int32_t* __restrict__ counts) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        atomicAdd(&counts[labels[i]], 1);
}

// Sort key: list id, then the row's score against its centroid (L2 distance,
// or -IP), so each list is ordered by ascending L2 / descending IP distance to
// the centroid as Index::add orders it (src/Index.cpp:643-651).
__global__ void sort_keys_kernel(const int64_t* __restrict__ labels, const float* __restrict__ score, int64_t n,
                                 uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float s = score[i];
        keys[i] = (static_cast<uint64_t>(labels[i]) << 32) | f2o(s);
        vals[i] = static_cast<int32_t>(i);
    }
}

// Place sorted row p into its list slot; write id and squared norm (the
// reference's candidate_norms, src/Index.cpp:689-696, sequential float sum).
__global__ void scatter_kernel(ArenaLayout L, const float* __restrict__ x, int64_t n, const int32_t* __restrict__ order,
                               const int64_t* __restrict__ labels, const int64_t* __restrict__ list_start,
                               const int64_t* __restrict__ list_off, const int32_t* __restrict__ keep,
                               float* __restrict__ codes, int64_t* __restrict__ ids, float* __restrict__ norms) {
    const int lane = threadIdx.x & 31;
    const int64_t p = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (p >= n) return;
    const int64_t src = order[p];
    const int64_t l = labels[src];
    if (keep && p - list_start[l] >= keep[l]) return;  // a list this index does not hold
    const int64_t r = list_off[l] + (p - list_start[l]);
    const float* xr = x + src * L.d;
    for (int b = 0; b < L.nb; ++b) {
        const int w = L.bstart[b + 1] - L.bstart[b];
        for (int j = lane; j < w; j += 32) codes[arena_offset(L, r, b, j)] = xr[L.bstart[b] + j];
    }
    if (lane == 0) {
        float s = 0.0f;
        for (int j = 0; j < L.d; ++j) s = __fadd_rn(s, __fmul_rn(xr[j], xr[j]));
        ids[r] = src;
        norms[r] = s;
    }
}

// Merge of `parts` per-query top-k lists (layout [parts][n][k], each sorted
// best first) into the best k: key (ordered score, part, rank), so equal
// distances keep the parts' order and then each part's own order.  One CTA
// per query.
__global__ void __launch_bounds__(256) merge_parts_kernel(const float* __restrict__ D, const int64_t* __restrict__ I,
                                                          int parts, int n, int k, int metric, float* __restrict__ oD,
                                                          int64_t* __restrict__ oI) {
    extern __shared__ __align__(16) unsigned char sm[];
    uint64_t* keys = reinterpret_cast<uint64_t*>(sm);
    const int q = blockIdx.x;
    const int total = parts * k;
    const int P = next_pow2(total);
    const bool l2 = metric == METRIC_L2;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        uint64_t key = KEY_MAX;
        if (i < total) {
            const int p = i / k, r = i % k;
            const size_t at = (static_cast<size_t>(p) * n + q) * k + r;
            if (I[at] >= 0) {
                const float sc = l2 ? D[at] : -D[at];
                key = (static_cast<uint64_t>(f2o(sc)) << 32) | (static_cast<uint32_t>(p) << 16) | static_cast<uint32_t>(r);
            }
        }
        keys[i] = key;
    }
    __syncthreads();
    cta_bitonic_sort(keys, P);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const uint64_t key = keys[i];
        const size_t o = static_cast<size_t>(q) * k + i;
        if (key == KEY_MAX) {
            oD[o] = l2 ? FLT_MAX : -FLT_MAX;
            oI[o] = -1;
        } else {
            const int p = static_cast<int>((key >> 16) & 0xffffu), r = static_cast<int>(key & 0xffffu);
            const size_t at = (static_cast<size_t>(p) * n + q) * k + r;
            oD[o] = D[at];
            oI[o] = I[at];
        }
    }
}

__global__ void fill_i64_kernel(int64_t* p, int64_t n, int64_t v) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        p[i] = v;
}

__global__ void gather_rows_kernel(const float* __restrict__ x, const int64_t* __restrict__ rows, int64_t n, int d,
                                   float* __restrict__ out) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n * d;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t r = i / d, j = i % d;
        out[i] = x[rows[r] * d + j];
    }
}

// Rows divided by their L2 norm (sequential float sum), zero rows unchanged
// (Eigen's colwise().normalized(), src/Clustering.cpp:122).
__global__ void normalize_rows_kernel(const float* __restrict__ x, int64_t n, int d, float* __restrict__ out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const float* xr = x + i * d;
    float s = 0.0f;
    for (int j = 0; j < d; ++j) s = __fadd_rn(s, __fmul_rn(xr[j], xr[j]));
    const float nr = sqrtf(s);
    for (int j = 0; j < d; ++j) out[i * d + j] = nr > 0.0f ? __fdiv_rn(xr[j], nr) : xr[j];
}

// FP64 accumulation of each row into its centroid's sum (one warp per row).
__global__ void kmeans_accumulate_kernel(const float* __restrict__ x, const int64_t* __restrict__ labels, int64_t n,
                                         int d, double* __restrict__ sums, unsigned long long* __restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const int64_t i = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    const int64_t l = labels[i];
    for (int j = lane; j < d; j += 32) atomicAdd(&sums[l * d + j], static_cast<double>(x[i * d + j]));
    if (lane == 0) atomicAdd(&counts[l], 1ull);
}

// Non-empty centroids become the mean of their rows; empty ones keep their
// previous value (src/Clustering.cpp:146-150).
__global__ void kmeans_update_kernel(const double* __restrict__ sums, const unsigned long long* __restrict__ counts,
                                     int nlist, int d, float* __restrict__ cent) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<int64_t>(nlist) * d) return;
    const unsigned long long c = counts[i / d];
    if (c > 0) cent[i] = static_cast<float>(sums[i] / static_cast<double>(c));
}

// IP centroids are L2-normalised after training (src/Index.cpp:408-419).
__global__ void normalize_centroids_kernel(float* cent, int nlist, int d) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nlist) return;
    float* v = cent + static_cast<size_t>(c) * d;
    float s = 0.0f;
    for (int j = 0; j < d; ++j) s = __fadd_rn(s, __fmul_rn(v[j], v[j]));
    if (s != 0.0f) {
        const float r = sqrtf(s);
        for (int j = 0; j < d; ++j) v[j] = __fdiv_rn(v[j], r);
    }
}

__global__ void unpack_list_kernel(ArenaLayout L, const float* __restrict__ codes, int64_t row0, int n,
                                   float* __restrict__ out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<int64_t>(n) * L.d) return;
    const int64_t r = i / L.d;
    const int j = static_cast<int>(i % L.d);
    int b = 0;
    while (b + 1 < L.nb && j >= L.bstart[b + 1]) ++b;
    out[i] = codes[arena_offset(L, row0 + r, b, j - L.bstart[b])];
}

inline int grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    if (g > (1 << 30)) g = 1 << 30;
    return static_cast<int>(g < 1 ? 1 : g);
}

}  // namespace

cudaError_t launch_coarse_scores(const float* q, int nq, const float* cent, int nlist, int d, int metric, float* out,
                                 cudaStream_t s) {
    dim3 grid((nlist + 63) / 64, (nq + 63) / 64);
    if (metric == METRIC_L2)
        coarse_scores_kernel<METRIC_L2><<<grid, 256, 0, s>>>(q, nq, cent, nlist, d, out);
    else
        coarse_scores_kernel<METRIC_IP><<<grid, 256, 0, s>>>(q, nq, cent, nlist, d, out);
    return cudaGetLastError();
}

cudaError_t launch_select(const float* scores, int nq, int n, int m, int64_t* out_idx, float* out_score,
                          cudaStream_t s) {
    if (m <= 256 && n <= 1024) {
        select_warp_kernel<32><<<(nq + 7) / 8, 256, 0, s>>>(scores, nq, n, m, out_idx, out_score);
        return cudaGetLastError();
    }
    if (m <= 256 && n <= 2048) {
        select_warp_kernel<64><<<(nq + 7) / 8, 256, 0, s>>>(scores, nq, n, m, out_idx, out_score);
        return cudaGetLastError();
    }
    const size_t smem = static_cast<size_t>(next_pow2(m)) * 8 + static_cast<size_t>(n) * 4;
    cudaError_t e = cudaFuncSetAttribute(select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    select_kernel<<<nq, 256, smem, s>>>(scores, n, m, out_idx, out_score);
    return cudaGetLastError();
}

cudaError_t launch_argmin(const float* scores, int nrows, int n, int64_t* out_idx, float* out_score,
                          cudaStream_t s) {
    argmin_kernel<<<grid_for(static_cast<int64_t>(nrows) * 32, 256), 256, 0, s>>>(scores, nrows, n, out_idx,
                                                                                  out_score);
    return cudaGetLastError();
}

cudaError_t launch_warmup(const ArenaLayout& L, const float* codes, const int64_t* list_off,
                          const int32_t* list_size, const float* q, int nq, const int64_t* probes, int nprobe, int k,
                          int wl, int wls, int blockwise, uint32_t* out_thr, float* out_f, int* err, cudaStream_t s,
                          int skip_lo, int skip_hi) {
    (void)err;
    const int wle = wl < nprobe ? wl : nprobe;
    cudaError_t e;
    if (wle <= 32 && static_cast<int64_t>(wle) * wls <= 1024) {
        const size_t wsmem = static_cast<size_t>(8) * L.row_pitch * 4;
        if ((e = cudaFuncSetAttribute(warmup_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(wsmem))) != cudaSuccess)
            return e;
        warmup_warp_kernel<<<(nq + 7) / 8, 256, wsmem, s>>>(L, codes, list_off, list_size, q, probes, nq, nprobe, k,
                                                            wl, wls, blockwise, out_thr, out_f, skip_lo, skip_hi);
        return cudaGetLastError();
    }
    const size_t smem = static_cast<size_t>(L.row_pitch) * 4 + static_cast<size_t>((wl + 2) & ~1) * 4 +
                        static_cast<size_t>(wl) * 8 + static_cast<size_t>(wle) * wls * 4;
    if ((e = cudaFuncSetAttribute(warmup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)) !=
        cudaSuccess)
        return e;
    warmup_kernel<<<nq, 256, smem, s>>>(L, codes, list_off, list_size, q, probes, nprobe, k, wl, wls, blockwise,
                                        out_thr, out_f, skip_lo, skip_hi);
    return cudaGetLastError();
}

template <int KR, int S>
static cudaError_t launch_scan_t(const ScanParams& p, int W, int* smem_out, cudaStream_t s) {
    const int npa = ((p.nprobe + p.nsplit - 1) / p.nsplit + 3) & ~3;
    const size_t smem = static_cast<size_t>(W) * S * 32 * p.L.max_pitch * 4 + static_cast<size_t>(W) * S * 8 +
                        static_cast<size_t>(W) * 2 * KR * 32 * 8 + static_cast<size_t>(KR) * 32 * 8 +
                        static_cast<size_t>(npa) * 8 +
                        static_cast<size_t>(p.L.row_pitch) * 4 + static_cast<size_t>(npa) * 8;
    if (smem_out) *smem_out = static_cast<int>(smem);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(scan_plain_kernel<KR, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    // With a device count and a query grid, the CTAs loop over the queries.
    const int gq = (p.nq_dev && p.qgrid > 0) ? std::min(p.nq, p.qgrid) : p.nq;
    if (gq < 1) return cudaSuccess;
    scan_plain_kernel<KR, S><<<gq * p.nsplit, W * 32, smem, s>>>(p);
    return cudaGetLastError();
}

// Warps, slots and K' are chosen so that one CTA's shared memory fits: 16
// warps with 2 slots each for pitches up to 32 floats per block (d <= 128
// with 4 blocks), 8 warps for wider blocks.  Slots are processed in pairs.
cudaError_t launch_scan_plain(const ScanParams& p, int* smem_out, cudaStream_t s) {
    const int kr = p.k <= 32 ? 1 : p.k <= 64 ? 2 : p.k <= 128 ? 4 : 8;
    const int slot_kb = p.L.max_pitch / 8;  // 32 rows x pitch floats, in KiB
    const int W = slot_kb * 2 * 16 <= 128 ? 16 : slot_kb * 2 * 8 <= 160 ? 8 : 4;
#define HY_SCAN_CASE(KR) \
    case KR:             \
        return launch_scan_t<KR, 2>(p, W, smem_out, s);
    switch (kr) {
        HY_SCAN_CASE(1)
        HY_SCAN_CASE(2)
        HY_SCAN_CASE(4)
        HY_SCAN_CASE(8)
        default:
            return cudaErrorInvalidValue;
    }
#undef HY_SCAN_CASE
}

cudaError_t launch_merge(const uint64_t* parts, int nq, int nparts, int kp, int k, int metric, const int64_t* ids,
                         float* D, int64_t* I, cudaStream_t s, int64_t* rows, const int32_t* nq_dev) {
    const size_t smem = nparts > 1 ? static_cast<size_t>(next_pow2(nparts * kp)) * 8 : 0;
    cudaError_t e = cudaFuncSetAttribute(merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    // With a device count the grid is capped and the CTAs loop over queries.
    const int grid = nq_dev ? std::min(nq, 1024) : nq;
    if (grid < 1) return cudaSuccess;
    merge_kernel<<<grid, 256, smem, s>>>(parts, nq, nparts, kp, k, metric, ids, D, I, rows, nq_dev);
    return cudaGetLastError();
}

cudaError_t launch_histogram(const int64_t* labels, int64_t n, int32_t* counts, cudaStream_t s) {
    histogram_kernel<<<grid_for(n, 256), 256, 0, s>>>(labels, n, counts);
    return cudaGetLastError();
}

cudaError_t launch_make_sort_keys(const int64_t* labels, const float* score, int64_t n, uint64_t* keys,
                                  int32_t* vals, cudaStream_t s) {
    sort_keys_kernel<<<grid_for(n, 256), 256, 0, s>>>(labels, score, n, keys, vals);
    return cudaGetLastError();
}

cudaError_t radix_sort_pairs(void* tmp, size_t* tmp_bytes, const uint64_t* kin, uint64_t* kout, const int32_t* vin,
                             int32_t* vout, int64_t n, int end_bit, cudaStream_t s) {
    return cub::DeviceRadixSort::SortPairs(tmp, *tmp_bytes, kin, kout, vin, vout, static_cast<int>(n), 0, end_bit, s);
}

cudaError_t launch_scatter(const ArenaLayout& L, const float* x, int64_t n, const int32_t* order,
                           const int64_t* labels, const int64_t* list_start, const int64_t* list_off,
                           const int32_t* keep, float* codes, int64_t* ids, float* norms, cudaStream_t s) {
    scatter_kernel<<<grid_for(n * 32, 256), 256, 0, s>>>(L, x, n, order, labels, list_start, list_off, keep, codes,
                                                         ids, norms);
    return cudaGetLastError();
}

cudaError_t launch_merge_parts(const float* D, const int64_t* I, int parts, int n, int k, int metric, float* oD,
                               int64_t* oI, cudaStream_t s) {
    const size_t smem = static_cast<size_t>(next_pow2(parts * k)) * 8;
    cudaError_t e = cudaFuncSetAttribute(merge_parts_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    merge_parts_kernel<<<n, 256, smem, s>>>(D, I, parts, n, k, metric, oD, oI);
    return cudaGetLastError();
}

cudaError_t launch_fill_i64(int64_t* p, int64_t n, int64_t v, cudaStream_t s) {
    fill_i64_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t launch_gather_rows(const float* x, const int64_t* rows, int64_t n, int d, float* out, cudaStream_t s) {
    gather_rows_kernel<<<grid_for(n * d, 256), 256, 0, s>>>(x, rows, n, d, out);
    return cudaGetLastError();
}

cudaError_t launch_normalize_rows(const float* x, int64_t n, int d, float* out, cudaStream_t s) {
    normalize_rows_kernel<<<grid_for(n, 128), 128, 0, s>>>(x, n, d, out);
    return cudaGetLastError();
}

cudaError_t launch_kmeans_accumulate(const float* x, const int64_t* labels, int64_t n, int d, double* sums,
                                     unsigned long long* counts, cudaStream_t s) {
    kmeans_accumulate_kernel<<<grid_for(n * 32, 256), 256, 0, s>>>(x, labels, n, d, sums, counts);
    return cudaGetLastError();
}

cudaError_t launch_kmeans_update(const double* sums, const unsigned long long* counts, int nlist, int d,
                                 float* cent, cudaStream_t s) {
    kmeans_update_kernel<<<grid_for(static_cast<int64_t>(nlist) * d, 256), 256, 0, s>>>(sums, counts, nlist, d,
                                                                                        cent);
    return cudaGetLastError();
}

cudaError_t launch_normalize_centroids(float* cent, int nlist, int d, cudaStream_t s) {
    normalize_centroids_kernel<<<grid_for(nlist, 128), 128, 0, s>>>(cent, nlist, d);
    return cudaGetLastError();
}

cudaError_t launch_unpack_list(const ArenaLayout& L, const float* codes, int64_t row0, int n, float* out,
                               cudaStream_t s) {
    unpack_list_kernel<<<grid_for(static_cast<int64_t>(n) * L.d, 256), 256, 0, s>>>(L, codes, row0, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Learned probe predictor: features, stop labels, per-query nprobe.
namespace {

// Features of one query from its P best centroid scores (ascending): f0 =
// log|s0|, fi = log1p((si - s0) / |s0|) for the next 63 (the last score is
// repeated when P < 64); then standardised with the model's mean and std.
__global__ void probe_features_kernel(const float* __restrict__ scores, int n, int P, const float* __restrict__ mu,
                                      const float* __restrict__ sd, float* __restrict__ X) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<int64_t>(n) * 64) return;
    const int64_t q = i / 64;
    const int f = static_cast<int>(i % 64);
    const float* sc = scores + q * P;
    const float s0 = sc[0];
    const float a0 = fabsf(s0) + 1e-6f;
    float v;
    if (f == 0)
        v = logf(a0);
    else
        v = log1pf(fmaxf(sc[min(f, P - 1)] - s0, 0.0f) / a0);
    X[i] = mu ? (v - mu[f]) / sd[f] : v;
}

// Stop label of each query: 1 + the largest probe rank among the lists that
// hold its exact top-kl rows (arena rows from the merge), i.e. the smallest
// nprobe whose lists contain all of them.
__global__ void stop_labels_kernel(const int64_t* __restrict__ rows, int n, int kl, const int64_t* __restrict__ probes,
                                   int P, const int64_t* __restrict__ list_off, int nlist, float* __restrict__ label) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int worst = 0;
    for (int i = 0; i < kl; ++i) {
        const int64_t r = rows[static_cast<int64_t>(q) * kl + i];
        if (r < 0) continue;
        int lo = 0, hi = nlist - 1;  // list = last l with list_off[l] <= r
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (list_off[mid] <= r)
                lo = mid;
            else
                hi = mid - 1;
        }
        int rank = P - 1;
        for (int j = 0; j < P; ++j)
            if (probes[static_cast<int64_t>(q) * P + j] == lo) {
                rank = j;
                break;
            }
        worst = max(worst, rank);
    }
    label[q] = static_cast<float>(worst + 1);
}

__global__ void cut_probes_kernel(int64_t* __restrict__ probes, int n, int P, const int32_t* __restrict__ np) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int c = max(1, min(P, np[q]));
    for (int j = c; j < P; ++j) probes[static_cast<int64_t>(q) * P + j] = -1;
}

// Per-query nprobe = clamp(ceil(2^(y + margin)), 1, P); probes beyond it
// become -1.  Adds the chosen counts to *total.
__global__ void apply_nprobe_kernel(const float* __restrict__ y, int n, float margin, int P,
                                    int64_t* __restrict__ probes, unsigned long long* __restrict__ total) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float e = exp2f(fminf(y[q] + margin, 30.0f));
    int np = static_cast<int>(ceilf(e));
    np = max(1, min(P, np));
    for (int j = np; j < P; ++j) probes[static_cast<int64_t>(q) * P + j] = -1;
    atomicAdd(total, static_cast<unsigned long long>(np));
}

}  // namespace

cudaError_t launch_cut_probes(int64_t* probes, int n, int P, const int32_t* np, cudaStream_t s) {
    cut_probes_kernel<<<grid_for(n, 128), 128, 0, s>>>(probes, n, P, np);
    return cudaGetLastError();
}

cudaError_t launch_probe_features(const float* scores, int n, int P, const float* mu, const float* sd, float* X,
                                  cudaStream_t s) {
    probe_features_kernel<<<grid_for(static_cast<int64_t>(n) * 64, 256), 256, 0, s>>>(scores, n, P, mu, sd, X);
    return cudaGetLastError();
}

cudaError_t launch_stop_labels(const int64_t* rows, int n, int kl, const int64_t* probes, int P,
                               const int64_t* list_off, int nlist, float* label, cudaStream_t s) {
    stop_labels_kernel<<<grid_for(n, 128), 128, 0, s>>>(rows, n, kl, probes, P, list_off, nlist, label);
    return cudaGetLastError();
}

cudaError_t launch_apply_nprobe(const float* y, int n, float margin, int P, int64_t* probes,
                                unsigned long long* total, cudaStream_t s) {
    apply_nprobe_kernel<<<grid_for(n, 128), 128, 0, s>>>(y, n, margin, P, probes, total);
    return cudaGetLastError();
}

}  // namespace hy
