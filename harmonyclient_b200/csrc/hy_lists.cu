// List-major exact FP32 scan (the plain form for batches in which lists are
// shared by several queries) and the per-query top-k steps around it.
//
// The reference scans query by query: each (query, probed list) pair streams
// the list's rows once (src/IVFScan.hpp:240-288, src/node.cpp:606-678).  Here
// the (query, probed list) pairs are inverted into per-list groups of up to
// 32 queries (the same work items as the tensor-core forms) and a persistent
// kernel drains the items: per item the CTA stages the group's queries in
// shared memory, and each warp streams 32-row tiles of the item's row slice,
// one dimension block at a time, through a ring of bulk copies.  A staged
// block is read into registers once (lane = row) and every query of the
// group that still has a live row in the tile accumulates against it, so a
// list's bytes are read once per group instead of once per query and the
// scan is bound by FP32 issue rather than by HBM.
//
// Arithmetic and pruning are the plain scan's: each dimension block is summed
// from zero in dimension order with separately rounded sub / mul / add, and
// block sums are added in order (src/node.cpp:646-650), so every distance is
// bit-identical to the query-major kernel's and the oracle's.  After each
// block but the last, a (row, query) pair whose partial sum exceeds the
// query's threshold is dropped (L2 only, as in the reference); a tile whose
// pairs are all dropped loads no further blocks.  At the last block, pairs
// with score <= threshold are appended to the query's candidate buffer as
// 64-bit keys (ordered score << 32 | arena row).
//
// Thresholds: the warm-up threshold (src/Index.cpp:999-1051) bounds a first
// pass over each query's nearest list; a warp-per-query step then keeps the
// k best keys and lowers the threshold to the k-th; a second pass scans the
// remaining probed lists under it; the final step sorts each query's
// candidates and writes the k best (distance, id), which are the query-major
// scan's answer.  A query whose candidates overflow the buffer is answered
// again by the query-major scan.
#include <algorithm>
#include <cfloat>
#include <cstddef>

#include "hy_common.cuh"
#include "hy_lists.cuh"

namespace hy {
namespace {

constexpr int METRIC_L2 = 1;  // include/hy.h's HY_METRIC_L2
constexpr int LM_WARPS = 8;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Decode work item g: {list, query group, row slice}.  Items beyond the
// descriptor table's capacity are found by a binary search over item_off.
__device__ inline int4 decode_item(const ListScanParams& p, int64_t g) {
    if (g < p.item_cap) return p.items[g];
    int lo = 0, hi = p.nlist - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (p.item_off[mid + 1] > g)
            hi = mid;
        else
            lo = mid + 1;
    }
    const int nrs = max(1, (p.list_size[lo] + p.rs - 1) / p.rs);
    const int w = static_cast<int>(g - p.item_off[lo]);
    return make_int4(lo, w / nrs, w % nrs, 0);
}

// One dimension block of one 32-row tile against the group's live queries.
// `rowp`: this lane's row of the staged block (pitch P floats); `qb(qi)`:
// query qi's block.  sp[qi] accumulates the block sums in order.
// MULTI = false: the block is one 32-float chunk group (pitch 32).
template <int QG, bool MULTI>
__device__ __forceinline__ void block_compute(const float* rowp, const float* qs, int row_pitch, int boff, int P,
                                              bool first, bool l2, uint32_t live, float (&sp)[QG], int lane) {
    if (!MULTI) {
        float4 xr[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) xr[c] = *reinterpret_cast<const float4*>(rowp + 4 * (c ^ (lane & 7)));
#pragma unroll
        for (int qi = 0; qi < QG; ++qi) {
            if (live & (1u << qi)) {
                const float* qb = qs + qi * row_pitch + boff;
                float a = 0.0f;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const float4 y = *reinterpret_cast<const float4*>(qb + 4 * c);
                    if (l2) {
                        a = sq_add(a, y.x, xr[c].x);
                        a = sq_add(a, y.y, xr[c].y);
                        a = sq_add(a, y.z, xr[c].z);
                        a = sq_add(a, y.w, xr[c].w);
                    } else {
                        a = ip_add(a, y.x, xr[c].x);
                        a = ip_add(a, y.y, xr[c].y);
                        a = ip_add(a, y.z, xr[c].z);
                        a = ip_add(a, y.w, xr[c].w);
                    }
                }
                sp[qi] = first ? a : __fadd_rn(sp[qi], a);
            }
        }
    } else {
        float acc[QG];
#pragma unroll
        for (int qi = 0; qi < QG; ++qi) acc[qi] = 0.0f;
        for (int s8 = 0; s8 < (P >> 2); s8 += 8) {
            float4 xr[8];
#pragma unroll
            for (int c = 0; c < 8; ++c)
                xr[c] = *reinterpret_cast<const float4*>(rowp + 4 * (s8 + (c ^ (lane & 7))));
#pragma unroll
            for (int qi = 0; qi < QG; ++qi) {
                if (live & (1u << qi)) {
                    const float* qb = qs + qi * row_pitch + boff + 4 * s8;
                    float a = acc[qi];
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const float4 y = *reinterpret_cast<const float4*>(qb + 4 * c);
                        if (l2) {
                            a = sq_add(a, y.x, xr[c].x);
                            a = sq_add(a, y.y, xr[c].y);
                            a = sq_add(a, y.z, xr[c].z);
                            a = sq_add(a, y.w, xr[c].w);
                        } else {
                            a = ip_add(a, y.x, xr[c].x);
                            a = ip_add(a, y.y, xr[c].y);
                            a = ip_add(a, y.z, xr[c].z);
                            a = ip_add(a, y.w, xr[c].w);
                        }
                    }
                    acc[qi] = a;
                }
            }
        }
#pragma unroll
        for (int qi = 0; qi < QG; ++qi)
            if (live & (1u << qi)) sp[qi] = first ? acc[qi] : __fadd_rn(sp[qi], acc[qi]);
    }
}

// Chunks [C0, C1) (4 dimensions each) of one query's block sum (qb: its 32
// block values) against this lane's row (xr), continuing from a, in
// dimension order; and of two queries at once, as two independent
// dependency chains.
template <bool L2, int C0, int C1>
__device__ __forceinline__ float chain1(const float* qb, const float4 (&xr)[8], float a) {
#pragma unroll
    for (int c = C0; c < C1; ++c) {
        const float4 y = *reinterpret_cast<const float4*>(qb + 4 * c);
        if (L2) {
            a = sq_add(a, y.x, xr[c].x);
            a = sq_add(a, y.y, xr[c].y);
            a = sq_add(a, y.z, xr[c].z);
            a = sq_add(a, y.w, xr[c].w);
        } else {
            a = ip_add(a, y.x, xr[c].x);
            a = ip_add(a, y.y, xr[c].y);
            a = ip_add(a, y.z, xr[c].z);
            a = ip_add(a, y.w, xr[c].w);
        }
    }
    return a;
}

template <bool L2, int C0, int C1>
__device__ __forceinline__ void chain2(const float* qa, const float* qb, const float4 (&xr)[8], float& a0,
                                       float& a1) {
    float s0 = a0, s1 = a1;
#pragma unroll
    for (int c = C0; c < C1; ++c) {
        const float4 y0 = *reinterpret_cast<const float4*>(qa + 4 * c);
        const float4 y1 = *reinterpret_cast<const float4*>(qb + 4 * c);
        if (L2) {
            s0 = sq_add(s0, y0.x, xr[c].x);
            s1 = sq_add(s1, y1.x, xr[c].x);
            s0 = sq_add(s0, y0.y, xr[c].y);
            s1 = sq_add(s1, y1.y, xr[c].y);
            s0 = sq_add(s0, y0.z, xr[c].z);
            s1 = sq_add(s1, y1.z, xr[c].z);
            s0 = sq_add(s0, y0.w, xr[c].w);
            s1 = sq_add(s1, y1.w, xr[c].w);
        } else {
            s0 = ip_add(s0, y0.x, xr[c].x);
            s1 = ip_add(s1, y1.x, xr[c].x);
            s0 = ip_add(s0, y0.y, xr[c].y);
            s1 = ip_add(s1, y1.y, xr[c].y);
            s0 = ip_add(s0, y0.z, xr[c].z);
            s1 = ip_add(s1, y1.z, xr[c].z);
            s0 = ip_add(s0, y0.w, xr[c].w);
            s1 = ip_add(s1, y1.w, xr[c].w);
        }
    }
    a0 = s0;
    a1 = s1;
}

// Persistent list-major scan.  QG queries per group (<= 32), R bulk-copy
// slots per warp, LM_WARPS warps.  Blocks of pitch 32 (MULTI = false) keep
// each (query, row) partial sum in shared memory and walk the live queries of
// a tile two at a time; wider blocks keep them in registers.
template <int QG, int R, bool MULTI, bool L2>
__global__ void __launch_bounds__(LM_WARPS * 32, MULTI ? 1 : 2)
    list_scan_kernel(const __grid_constant__ ListScanParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const ArenaLayout& L = p.L;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t slot_floats = static_cast<size_t>(32) * L.max_pitch;
    float* bufs = reinterpret_cast<float*>(smem);
    float* qs = bufs + static_cast<size_t>(LM_WARPS) * R * slot_floats;
    float* sps = qs + static_cast<size_t>(QG) * L.row_pitch;  // [warp][query][lane] partial sums (pitch 32)
    uint64_t* bars = reinterpret_cast<uint64_t*>(sps + (MULTI ? 0 : static_cast<size_t>(LM_WARPS) * QG * 32));
    __shared__ float s_thr[QG];
    __shared__ float s_lo[QG], s_hi[QG];  // OPT_TRIANGLE: each query's candidate2centroid window
    __shared__ int s_qid[QG];
    __shared__ int s_next, s_ntiles, s_nrows, s_nqv, s_done, s_list;
    __shared__ long long s_row0;
    // The next item, claimed and described by warp 0 while the CTA scans the
    // current one (scalars only: two CTAs of the pitch-32 scan fill an SM's
    // shared memory to within a few hundred bytes).
    __shared__ int n_ntiles, n_nrows, n_nqv, n_done, n_list;
    __shared__ long long n_row0, n_pq, s_pq;
    // Per-warp ring tags: tile index within the item and block of each slot.
    __shared__ int s_tag_tile[LM_WARPS][R];
    __shared__ int s_tag_b[LM_WARPS][R];

    if (threadIdx.x == 0) {
        for (int i = 0; i < LM_WARPS * R; ++i) mbar_init(&bars[i], 1);
        fence_mbar_init();
    }
    float* wb = bufs + static_cast<size_t>(warp) * R * slot_floats;
    uint64_t* wbar = bars + warp * R;
    constexpr bool l2 = L2;
    const bool prune = p.prune && l2;
    float* spw = sps + static_cast<size_t>(warp) * QG * 32 + lane;
    uint32_t iss = 0, con = 0;  // copies issued / consumed by this warp (ring position)
    unsigned long long loaded = 0, computed = 0, possible = 0, possible_sums = 0;
    const int64_t nitems = p.item_off[p.nlist];

    // Lane 0 of warp 0: claim the next item and load its descriptor into
    // n_* (n_pq: the offset of its query ids in p.pairs).
    auto prefetch = [&]() {
        if (lane != 0) return;
        // No further items once a wait anywhere has given up.
        const unsigned int g = *reinterpret_cast<volatile int*>(p.err) ? 0xffffffffu : atomicAdd(p.work, 1u);
        if (g == 0xffffffffu || static_cast<int64_t>(g) >= nitems) {
            n_done = 1;
            return;
        }
        const int4 it = decode_item(p, g);
        const int l = it.x;
        const int lrow0 = it.z * p.rs;
        n_nqv = min(QG, p.pair_cnt[l] - it.y * QG);
        n_nrows = min(p.rs, p.list_size[l] - lrow0);
        n_ntiles = (n_nrows + 31) >> 5;
        n_row0 = p.list_off[l] + lrow0;
        n_list = l;
        n_pq = p.pair_off[l] + static_cast<int64_t>(it.y) * QG;
        n_done = 0;
    };
    if (warp == 0) prefetch();

    for (;;) {
        __syncthreads();  // previous item done, the next one prefetched (and, first time, barriers initialised)
        if (threadIdx.x == 0) {
            s_done = n_done;
            s_nqv = n_nqv;
            s_nrows = n_nrows;
            s_ntiles = n_ntiles;
            s_row0 = n_row0;
            s_list = n_list;
            s_pq = n_pq;
            s_next = 0;
        }
        __syncthreads();
        if (s_done) break;
        const int nqv = s_nqv;
        const int32_t* pq = p.pairs + s_pq;
        // Query ids and thresholds (score units; +inf when the query has none).
        if (threadIdx.x < QG) {
            const int j = threadIdx.x;
            const int qid = j < nqv ? pq[j] : -1;
            float t = -INFINITY;
            if (j < nqv) {
                const uint32_t key = p.thr ? p.thr[qid] : 0xffffffffu;
                t = key == 0xffffffffu ? INFINITY : o2f(key);
            }
            s_qid[j] = qid;
            s_thr[j] = t;
        }
        // The group's queries in the arena's block-padded layout.
        for (int i = threadIdx.x; i < QG * L.row_pitch; i += blockDim.x) {
            const int j = i / L.row_pitch, e = i - j * L.row_pitch;
            float v = 0.0f;
            if (j < nqv) {
                int b = 0;
                while (b + 1 < L.nb && e >= L.boff[b + 1]) ++b;
                const int w = L.bstart[b + 1] - L.bstart[b];
                const int jj = e - L.boff[b];
                // The query id from the pair list (s_qid is being written).
                if (jj < w) v = p.q[static_cast<size_t>(pq[j]) * L.d + L.bstart[b] + jj];
            }
            qs[i] = v;
        }
        if (p.triangle) {
            __syncthreads();  // s_qid and s_thr are read below
            const float* cl = p.cent + static_cast<size_t>(s_list) * L.d;
            for (int j = warp; j < QG; j += LM_WARPS) {
                float c = 0.0f;
                if (j < nqv) {
                    const float* qj = p.q + static_cast<size_t>(s_qid[j]) * L.d;
                    for (int e = lane; e < L.d; e += 32)
                        c = l2 ? __fmaf_rn(qj[e] - cl[e], qj[e] - cl[e], c) : __fmaf_rn(qj[e], cl[e], c);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
                }
                if (lane == 0) {
                    if (l2) {
                        // |q - x| >= | |q - c| - |x - c| |: a row whose distance
                        // to the centroid lies outside [rq - t, rq + t], t =
                        // sqrt(threshold), cannot reach the threshold.  Both
                        // ends are widened by relative margins far above the
                        // FP32 rounding of these norms and of the scan's
                        // sums, so no row the exact scan would admit is
                        // skipped.  No threshold: t = inf, nothing skipped.
                        const float rq = sqrtf(c);
                        const float t = sqrtf(s_thr[j]) * 1.0001f + rq * 1e-4f + 1e-6f;
                        s_lo[j] = (rq - t) * (1.0f - 2e-4f);
                        s_hi[j] = (rq + t) * (1.0f + 2e-4f);
                    } else {
                        // The reference's inner-product window
                        // (src/Index.cpp:1519-1542): with s = the query's k-th
                        // similarity so far and c = its inner product with
                        // the centroid, rows whose candidate2centroid lies
                        // outside [s c - sqrt(1-s^2) sqrt(1-c^2), s c +
                        // sqrt(1-s^2) sqrt(1-c^2)] (no upper limit when
                        // s < c) cannot reach s for unit-norm rows and
                        // queries.  Without a threshold (s = -inf) or off the
                        // unit sphere the bounds are NaN and nothing is
                        // skipped, as in the reference.
                        const float sim = -s_thr[j];
                        const float ss = sqrtf(1.0f - sim * sim), sc = sqrtf(1.0f - c * c);
                        s_lo[j] = sim * c - ss * sc;
                        s_hi[j] = sim < c ? INFINITY : sim * c + ss * sc;
                    }
                }
            }
        }
        __syncthreads();
        if (warp == 0) prefetch();  // the next item, while the other warps start on this one
        const int ntiles = s_ntiles, nrows = s_nrows;
        const int64_t row0 = s_row0;
        const uint32_t qmask = nqv >= 32 ? 0xffffffffu : ((1u << nqv) - 1u);

        // Issuer state (warp-uniform): the tile being issued and its next block.
        int it_tile = -1, it_b = 0;
        bool more = true;
        // Consumer state.
        int cur_tile = -1, dead_tile = -1;
        uint32_t alive = 0;
        float sp[QG];
#pragma unroll
        for (int qi = 0; qi < QG; ++qi) sp[qi] = 0.0f;

        auto refill = [&]() {
            while (iss - con < static_cast<uint32_t>(R)) {
                if (it_tile < 0) {
                    if (!more) return;
                    int g = 0;
                    if (lane == 0) g = atomicAdd(&s_next, 1);
                    g = __shfl_sync(FULL, g, 0);
                    if (g >= ntiles) {
                        more = false;
                        return;
                    }
                    possible += L.nb;
                    possible_sums += static_cast<unsigned long long>(L.row_pitch >> 4) * nqv;
                    if (p.triangle) {
                        // A tile whose rows lie outside every query's window
                        // is not loaded.
                        const float2 tr = p.c2c_tile[(row0 >> 5) + g];
                        const bool hit = lane < nqv && !(tr.y > s_hi[lane]) && !(tr.x < s_lo[lane]);
                        if (!__any_sync(FULL, hit)) continue;
                    }
                    it_tile = g;
                    it_b = 0;
                }
                const int slot = static_cast<int>(iss % R);
                const int b = it_b;
                const uint32_t bytes = static_cast<uint32_t>(32 * L.pitch[b] * sizeof(float));
                const float* src = p.codes + static_cast<size_t>((row0 >> 5) + it_tile) * 32 * L.row_pitch +
                                   static_cast<size_t>(L.boff[b]) * 32;
                if (lane == 0) {
                    s_tag_tile[warp][slot] = it_tile;
                    s_tag_b[warp][slot] = b;
                    fence_proxy_async();
                    mbar_expect_tx(&wbar[slot], bytes);
                    bulk_g2s(wb + static_cast<size_t>(slot) * slot_floats, src, bytes, &wbar[slot]);
                }
                ++iss;
                ++loaded;
                if (++it_b == L.nb) it_tile = -1;
            }
        };

        refill();
        __syncwarp();
        while (con != iss) {
            const int slot = static_cast<int>(con % R);
            const uint32_t parity = (con / R) & 1u;
            if (!mbar_wait_bounded(&wbar[slot], parity, p.err)) {
                // Give up on the item (the status word is raised); the
                // copies in flight are waited for below, bounded.
                more = false;
                it_tile = -1;
                ++con;
                for (; con != iss; ++con) mbar_wait_bounded(&wbar[con % R], (con / R) & 1u, p.err);
                break;
            }
            const int tile = s_tag_tile[warp][slot];
            const int b = s_tag_b[warp][slot];
            if (tile != cur_tile) {
                cur_tile = tile;
                const int nv = min(32, nrows - 32 * tile);
                alive = lane < nv ? qmask : 0u;
                if (p.triangle && lane < nv) {
                    const float cc = p.c2c[row0 + 32 * static_cast<int64_t>(tile) + lane];
#pragma unroll
                    for (int qi = 0; qi < QG; ++qi)
                        if (cc > s_hi[qi] || cc < s_lo[qi]) alive &= ~(1u << qi);
                }
            }
            if (tile != dead_tile) {
                const uint32_t live = __reduce_or_sync(FULL, alive);
                if (live == 0u) {
                    dead_tile = tile;
                    if (it_tile == tile) it_tile = -1;  // issue none of its further blocks
                } else if (!MULTI) {
                    const float* rowp = wb + static_cast<size_t>(slot) * slot_floats + lane * 32;
                    float4 xr[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        xr[c] = *reinterpret_cast<const float4*>(rowp + 4 * (c ^ (lane & 7)));
                    const float* qbase = qs + L.boff[b];
                    const bool first = b == 0, last = b + 1 == L.nb;
                    const int64_t arow = row0 + 32 * static_cast<int64_t>(tile) + lane;
                    // This block's sum of query qi is done: add it to the
                    // running partial, then prune or emit.
                    auto finish = [&](int qi, float a) {
                        const float sv = first ? a : __fadd_rn(spw[qi * 32], a);
                        if (!last) {
                            spw[qi * 32] = sv;
                            if (prune && sv > s_thr[qi]) alive &= ~(1u << qi);
                            return;
                        }
                        const float score = l2 ? sv : -sv;
                        const bool c = ((alive >> qi) & 1u) && score <= s_thr[qi];
                        const uint32_t bal = __ballot_sync(FULL, c);
                        if (bal) {
                            const int qid = s_qid[qi];
                            int base = 0;
                            if (lane == 0) base = atomicAdd(&p.cand_cnt[qid], __popc(bal));
                            base = __shfl_sync(FULL, base, 0);
                            const int pos = base + __popc(bal & lanemask_lt());
                            if (c && pos < p.capq)
                                p.cand[static_cast<size_t>(qid) * p.capq + pos] =
                                    (static_cast<uint64_t>(f2o(score)) << 32) | static_cast<uint32_t>(arow);
                        }
                    };
                    // After the first 16 dimensions: a query none of whose
                    // live rows can stay under its threshold (the partial,
                    // which only grows, already exceeds it) is dropped from
                    // the tile without the block's other 16 dimensions.
                    auto dead_here = [&](int qi, float a) -> bool {
                        const float lb = first ? a : __fadd_rn(spw[qi * 32], a);
                        return !((alive >> qi) & 1u) || lb > s_thr[qi];
                    };
                    auto half_dead = [&](int qi, float a) -> bool {
                        if (!prune) return false;
                        if (!__all_sync(FULL, dead_here(qi, a))) return false;
                        alive &= ~(1u << qi);
                        return true;
                    };
                    // Both queries of a pair in one warp reduction.
                    auto half_dead2 = [&](int qa, float a0, int qb, float a1, bool& da, bool& db) {
                        da = db = false;
                        if (!prune) return;
                        const unsigned m = (dead_here(qa, a0) ? 1u : 0u) | (dead_here(qb, a1) ? 2u : 0u);
                        const unsigned all = __reduce_and_sync(FULL, m);
                        da = (all & 1u) != 0u;
                        db = (all & 2u) != 0u;
                        if (da) alive &= ~(1u << qa);
                        if (db) alive &= ~(1u << qb);
                    };
                    uint32_t todo = live;
                    while (todo) {
                        const int qa = __ffs(todo) - 1;
                        todo &= todo - 1;
                        const float* ya = qbase + qa * L.row_pitch;
                        if (todo) {
                            const int qb = __ffs(todo) - 1;
                            todo &= todo - 1;
                            const float* yb = qbase + qb * L.row_pitch;
                            float a0 = 0.0f, a1 = 0.0f;
                            chain2<L2, 0, 4>(ya, yb, xr, a0, a1);
                            bool da, db;
                            half_dead2(qa, a0, qb, a1, da, db);
                            computed += 4 - (da ? 1 : 0) - (db ? 1 : 0);
                            if (!da && !db) {
                                chain2<L2, 4, 8>(ya, yb, xr, a0, a1);
                                finish(qa, a0);
                                finish(qb, a1);
                            } else if (!da) {
                                finish(qa, chain1<L2, 4, 8>(ya, xr, a0));
                            } else if (!db) {
                                finish(qb, chain1<L2, 4, 8>(yb, xr, a1));
                            }
                        } else {
                            const float a0 = chain1<L2, 0, 4>(ya, xr, 0.0f);
                            const bool da = half_dead(qa, a0);
                            computed += da ? 1 : 2;
                            if (!da) finish(qa, chain1<L2, 4, 8>(ya, xr, a0));
                        }
                    }
                } else {
                    computed += static_cast<unsigned long long>(__popc(live)) * (L.pitch[b] >> 4);
                    const int P = L.pitch[b];
                    const float* rowp = wb + static_cast<size_t>(slot) * slot_floats + lane * P;
                    block_compute<QG, MULTI>(rowp, qs, L.row_pitch, L.boff[b], P, b == 0, l2, live, sp, lane);
                    if (b + 1 < L.nb) {
                        if (prune) {
#pragma unroll
                            for (int qi = 0; qi < QG; ++qi)
                                if ((live & (1u << qi)) && sp[qi] > s_thr[qi]) alive &= ~(1u << qi);
                        }
                    } else {
                        const int64_t arow = row0 + 32 * static_cast<int64_t>(tile) + lane;
#pragma unroll
                        for (int qi = 0; qi < QG; ++qi) {
                            if (live & (1u << qi)) {
                                const float score = l2 ? sp[qi] : -sp[qi];
                                const bool c = ((alive >> qi) & 1u) && score <= s_thr[qi];
                                const uint32_t bal = __ballot_sync(FULL, c);
                                if (bal) {
                                    const int qid = s_qid[qi];
                                    int base = 0;
                                    if (lane == 0) base = atomicAdd(&p.cand_cnt[qid], __popc(bal));
                                    base = __shfl_sync(FULL, base, 0);
                                    const int pos = base + __popc(bal & lanemask_lt());
                                    if (c && pos < p.capq)
                                        p.cand[static_cast<size_t>(qid) * p.capq + pos] =
                                            (static_cast<uint64_t>(f2o(score)) << 32) | static_cast<uint32_t>(arow);
                                }
                            }
                        }
                    }
                }
            }
            __syncwarp();  // every lane is done with the slot before it is refilled
            ++con;
            refill();
            __syncwarp();
        }
    }
    if (lane == 0 && p.counters) {
        atomicAdd(&p.counters[0], loaded);
        atomicAdd(&p.counters[1], possible);
        atomicAdd(&p.counters[2], computed);
        atomicAdd(&p.counters[3], possible_sums);
    }
}

// Per query (one warp): the K' = 32 KR smallest candidate keys.  mode 0
// (after the first pass): the k best keys replace the buffer, the count
// becomes min(count, k) and the threshold drops to the k-th key's score when
// there are k.  mode 1 (final): the k best become (distance, id) rows of D / I
// (unfilled: the reference's heap_init values); a query whose candidates
// overflowed the buffer is listed in ovf (count, then query ids) instead.
template <int KR>
__global__ void __launch_bounds__(256) list_topk_kernel(uint64_t* __restrict__ cand, int32_t* __restrict__ cnt,
                                                        int nq, int capq, int k, int metric, int mode,
                                                        uint32_t* __restrict__ thr, const int64_t* __restrict__ ids,
                                                        float* __restrict__ D, int64_t* __restrict__ I,
                                                        int32_t* __restrict__ ovf) {
    constexpr int KP = KR * 32;
    const int lane = threadIdx.x & 31;
    const int q = static_cast<int>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (q >= nq) return;
    const int n = cnt[q];
    if (n > capq) {
        if (mode == 1 && lane == 0) {
            const int pos = atomicAdd(&ovf[0], 1);
            ovf[1 + pos] = q;
        }
        return;
    }
    uint64_t* c = cand + static_cast<size_t>(q) * capq;
    uint64_t t[KR];
#pragma unroll
    for (int r = 0; r < KR; ++r) t[r] = KEY_MAX;
    for (int base = 0; base < n; base += KP) {
        uint64_t v[KR];
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const int idx = base + r * 32 + lane;
            v[r] = idx < n ? c[idx] : KEY_MAX;
        }
        warp_sort<KR>(v, lane);
        warp_merge<KR>(t, v, lane);
    }
    if (mode == 0) {
        __syncwarp();
#pragma unroll
        for (int r = 0; r < KR; ++r) {
            const int e = r * 32 + lane;
            if (e < k && e < n) c[e] = t[r];
        }
        if (lane == 0) {
            cnt[q] = min(n, k);
        }
        if (n >= k) {
            const uint64_t kth = warp_get<KR>(t, k - 1);
            if (lane == 0) {
                const uint32_t key = static_cast<uint32_t>(kth >> 32);
                if (key < thr[q]) thr[q] = key;
            }
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < KR; ++r) {
        const int e = r * 32 + lane;
        if (e < k) {
            const uint64_t key = t[r];
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
            D[static_cast<size_t>(q) * k + e] = dv;
            I[static_cast<size_t>(q) * k + e] = iv;
        }
    }
}

// Per arena row: its inner product with its list's centroid (l2 = false; the
// reference's candidate2centroid, src/Index.cpp:659-667, by which a list is
// ordered, descending), or its L2 distance (not squared) to it (l2 = true; a
// list is ordered by it, ascending); and per 32-row tile {max, min} over its
// valid rows.  One warp per tile; lane = row.
__global__ void row_centroid_kernel(ArenaLayout L, const float* __restrict__ codes,
                                    const int64_t* __restrict__ list_off, const int32_t* __restrict__ list_size,
                                    int nlist, const float* __restrict__ cent, bool l2, float* __restrict__ c2c,
                                    float2* __restrict__ c2c_tile) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    // gw enumerates (list, tile of the list): find the list by binary search
    // over the tile offsets list_off / 32.
    const int64_t ntiles_all = list_off[nlist] >> 5;
    if (gw >= ntiles_all) return;
    int lo = 0, hi = nlist - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((list_off[mid] >> 5) <= gw)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int l = lo;
    const int64_t r = gw * 32 + lane;
    const bool valid = r - list_off[l] < list_size[l];
    float v = 0.0f;
    if (valid) {
        const float* c = cent + static_cast<size_t>(l) * L.d;
        for (int b = 0; b < L.nb; ++b) {
            const int w = L.bstart[b + 1] - L.bstart[b];
            for (int j = 0; j < w; ++j) {
                const float xv = codes[arena_offset(L, r, b, j)], cv = c[L.bstart[b] + j];
                v = l2 ? __fmaf_rn(xv - cv, xv - cv, v) : __fadd_rn(v, __fmul_rn(xv, cv));
            }
        }
        if (l2) v = sqrtf(v);
    }
    c2c[r] = v;
    float mx = valid ? v : -INFINITY, mn = valid ? v : INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
        mn = fminf(mn, __shfl_xor_sync(FULL, mn, o));
    }
    if (lane == 0) c2c_tile[gw] = make_float2(mx, mn);
}

template <int QG, int R, bool MULTI>
size_t list_scan_smem(const ArenaLayout& L) {
    return static_cast<size_t>(LM_WARPS) * R * 32 * L.max_pitch * 4 + static_cast<size_t>(QG) * L.row_pitch * 4 +
           (MULTI ? 0 : static_cast<size_t>(LM_WARPS) * QG * 32 * 4) + static_cast<size_t>(LM_WARPS) * R * 8;
}

template <int QG, int R, bool MULTI, bool L2>
cudaError_t launch_list_scan_m(const ListScanParams& p, int nsm, cudaStream_t s) {
    const size_t smem = list_scan_smem<QG, R, MULTI>(p.L);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    auto kern = list_scan_kernel<QG, R, MULTI, L2>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, LM_WARPS * 32, smem);
    if (e != cudaSuccess) return e;
    per_sm = std::max(1, per_sm);
    kern<<<nsm * per_sm, LM_WARPS * 32, smem, s>>>(p);
    return cudaGetLastError();
}

template <int QG, int R, bool MULTI>
cudaError_t launch_list_scan_t(const ListScanParams& p, int nsm, cudaStream_t s) {
    return p.metric == METRIC_L2 ? launch_list_scan_m<QG, R, MULTI, true>(p, nsm, s)
                                 : launch_list_scan_m<QG, R, MULTI, false>(p, nsm, s);
}

}  // namespace

bool list_scan_multi(const ArenaLayout& L) {
    for (int b = 0; b < L.nb; ++b)
        if (L.pitch[b] != 32) return true;
    return false;
}

bool list_scan_fits(const ArenaLayout& L) {
    if (!list_scan_multi(L)) return list_scan_smem<LM_GROUP, 2, false>(L) <= 227 * 1024;
    if (L.max_pitch <= 64) return list_scan_smem<LM_GROUP, 2, true>(L) <= 227 * 1024;
    return list_scan_smem<LM_GROUP, 1, true>(L) <= 227 * 1024;
}

cudaError_t launch_list_scan(const ListScanParams& p, int nsm, cudaStream_t s) {
    if (p.qg != LM_GROUP) return cudaErrorInvalidValue;
    // Pitch-32 blocks: two ring slots per warp (with the shared-memory
    // partial sums, two CTAs per SM); wider blocks: two slots while they fit
    // (pitch <= 64 floats), else one.
    if (!list_scan_multi(p.L)) return launch_list_scan_t<LM_GROUP, 2, false>(p, nsm, s);
    if (p.L.max_pitch <= 64) return launch_list_scan_t<LM_GROUP, 2, true>(p, nsm, s);
    return launch_list_scan_t<LM_GROUP, 1, true>(p, nsm, s);
}

cudaError_t launch_row_centroid(const ArenaLayout& L, const float* codes, const int64_t* list_off,
                                const int32_t* list_size, int nlist, int64_t arena_rows, const float* cent, int metric,
                                float* c2c, float2* c2c_tile, cudaStream_t s) {
    const int64_t tiles = arena_rows / 32;
    if (tiles < 1) return cudaSuccess;
    row_centroid_kernel<<<static_cast<int>((tiles * 32 + 255) / 256), 256, 0, s>>>(
        L, codes, list_off, list_size, nlist, cent, metric == METRIC_L2, c2c, c2c_tile);
    return cudaGetLastError();
}

cudaError_t launch_list_topk(uint64_t* cand, int32_t* cnt, int nq, int capq, int k, int metric, int mode,
                             uint32_t* thr, const int64_t* ids, float* D, int64_t* I, int32_t* ovf, cudaStream_t s) {
    const int kr = k <= 32 ? 1 : k <= 64 ? 2 : k <= 128 ? 4 : 8;
    const int grid = static_cast<int>((static_cast<int64_t>(nq) * 32 + 255) / 256);
    if (grid < 1) return cudaSuccess;
#define HY_TOPK_CASE(KR)                                                                                       \
    case KR:                                                                                                   \
        list_topk_kernel<KR><<<grid, 256, 0, s>>>(cand, cnt, nq, capq, k, metric, mode, thr, ids, D, I, ovf); \
        break;
    switch (kr) {
        HY_TOPK_CASE(1)
        HY_TOPK_CASE(2)
        HY_TOPK_CASE(4)
        HY_TOPK_CASE(8)
        default:
            return cudaErrorInvalidValue;
    }
#undef HY_TOPK_CASE
    return cudaGetLastError();
}

}  // namespace hy
