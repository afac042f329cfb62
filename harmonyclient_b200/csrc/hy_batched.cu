// Batched list-major scan on the tcgen05 tensor cores (the "bf16" form).
//
// Queries that probe the same list share one pass over it.  After coarse
// quantisation, the (query, probed list) pairs are inverted into per-list
// query groups; a persistent kernel (one CTA per SM) drains a work queue of
// (list, group of <=128 queries, slice of <=RS rows) items.  Per item the CTA
// gathers the group's bf16 query vectors into shared memory (the MMA's B
// operand), then streams the slice's 128-row tiles of the bf16 list arena
// (already stored in the tensor core's swizzled shared-memory image, so each
// 64-dimension k-block of a tile is one 16 KiB bulk copy) through a ring of
// stages.  One thread issues tcgen05.mma (M = 128 rows, N = 128 queries,
// K = 16) into one of two TMEM accumulators; four epilogue warps read the
// accumulator (thread = row), form dist = |x|^2 + |q|^2 - 2 q.x (or -q.x for
// inner product) and emit every (query, row) whose distance passes the
// query's threshold into that query's candidate buffer.  A final kernel
// re-ranks each query's best candidates with the exact FP32 distance (the
// plain scan's arithmetic) and writes the top-k.
//
// The threshold is an upper bound on the query's final k-th distance (the
// warm-up threshold), so no row of the exact top-k is rejected as long as its
// bf16 distance is not above it; on integer-valued data below 2^8 the bf16
// distances are exact.  A query whose candidates overflow its buffer is
// reported so the caller can answer it with the plain scan.
#include <cuda_bf16.h>

#include <cfloat>

#include "hy_batched.cuh"
#include "hy_common.cuh"
#include "hy_tc.cuh"

namespace hy {
namespace {

constexpr int QG = 128;      // queries per group (MMA N)
constexpr int TM = 128;      // rows per tile (MMA M)
constexpr int NS = 6;        // A stages (one 16 KiB k-block each)
constexpr int KB_BYTES = 16384;
constexpr int TMEM_COLS = 256;  // two accumulators of QG columns

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

// Per-row quantities for the bf16 error bound: |x~| (norm of the bf16-rounded
// row) and |x - x~| (its rounding error), one warp per arena row.
__global__ void row_aux_kernel(ArenaLayout L, const float* __restrict__ codes, int64_t rows, float2* __restrict__ aux) {
    const int lane = threadIdx.x & 31;
    const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (r >= rows) return;
    float nn = 0.0f, ee = 0.0f;
    for (int j = lane; j < L.d; j += 32) {
        int b = 0;
        while (b + 1 < L.nb && j >= L.bstart[b + 1]) ++b;
        const float v = codes[arena_offset(L, r, b, j - L.bstart[b])];
        const float vb = __bfloat162float(__float2bfloat16_rn(v));
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

// Queries: bf16 rows padded to nkb*64, and per query {|q|^2 (sequential f32,
// the exact arithmetic's value), |q|, |q~|, |q - q~|}.
__global__ void prep_queries_kernel(const float* __restrict__ q, int nq, int d, int nkb,
                                    __nv_bfloat16* __restrict__ qb, float4* __restrict__ qaux) {
    const int i = blockIdx.x;
    if (i >= nq) return;
    const float* src = q + static_cast<size_t>(i) * d;
    float nn = 0.0f, ee = 0.0f;
    for (int j = threadIdx.x; j < nkb * 64; j += blockDim.x) {
        const float v = j < d ? src[j] : 0.0f;
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        qb[static_cast<size_t>(i) * nkb * 64 + j] = b;
        const float vb = __bfloat162float(b);
        nn = fmaf(vb, vb, nn);
        ee = fmaf(v - vb, v - vb, ee);
    }
    __shared__ float red[2][4];
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
    }
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
__global__ void probe_hist_kernel(const int64_t* __restrict__ probes, int64_t n, int32_t* __restrict__ cnt) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t l = probes[i];
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

__global__ void probe_fill_kernel(const int64_t* __restrict__ probes, int nq, int nprobe,
                                  const int64_t* __restrict__ off, int32_t* __restrict__ fill,
                                  int32_t* __restrict__ pairs) {
    const int64_t n = static_cast<int64_t>(nq) * nprobe;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t l = probes[i];
        if (l < 0) continue;
        const int pos = atomicAdd(&fill[l], 1);
        pairs[off[l] + pos] = static_cast<int32_t>(i / nprobe);
    }
}

// Items of a list = query groups x row slices (none for an empty list).
__global__ void item_count_kernel(const int32_t* __restrict__ cnt, const int32_t* __restrict__ list_size, int nlist,
                                  int rs, int32_t* __restrict__ items) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlist) return;
    const int c = cnt[l], s = list_size[l];
    items[l] = (c > 0 && s > 0) ? ((c + QG - 1) / QG) * ((s + rs - 1) / rs) : 0;
}

// ---------------------------------------------------------------------------
struct BatchedParams {
    const unsigned char* abf;       // bf16 arena image
    const int64_t* list_off;        // [nlist+1]
    const int32_t* list_size;       // [nlist]
    const int64_t* item_off;        // [nlist+1]
    const int64_t* pair_off;        // [nlist+1]
    const int32_t* pairs;           // query ids grouped by list
    const int32_t* pair_cnt;        // [nlist]
    const float* xn;                // [arena rows] squared norms (f32)
    const float2* xaux;             // [arena rows] {|x~|, |x - x~|}
    const __nv_bfloat16* qb;        // [nq][nkb*64]
    const float4* qaux;             // [nq] {|q|^2, |q|, |q~|, |q - q~|}
    const float* thr;               // [nq] distance thresholds (score units)
    uint64_t* cand;                 // [nq][capq]
    int32_t* cand_cnt;              // [nq]
    unsigned int* work;             // work-queue counter
    int* err;
    int nlist, nkb, rs, capq, metric;
    float cK, cN;                   // error-bound constants (see err_coef)
};

__global__ void __launch_bounds__(256, 1) batched_scan_kernel(const __grid_constant__ BatchedParams p) {
    extern __shared__ unsigned char sm_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sB = base;                                   // nkb x 16 KiB (queries)
    unsigned char* sA = sB + static_cast<size_t>(p.nkb) * KB_BYTES;  // NS x 16 KiB (list k-blocks)
    __shared__ uint64_t full[NS], empty[NS], accf[2], acce[2];
    __shared__ uint32_t tbase;
    __shared__ float s_qn[QG], s_thr[QG], s_aq[QG], s_bq[QG];
    __shared__ int s_qid[QG];
    constexpr int CB = 256;  // per-epilogue-warp candidate staging
    __shared__ int s_cq[4][CB];
    __shared__ uint64_t s_ck[4][CB];
    // Two item descriptors: the one being processed and the next one, which
    // warp 2 fetches and decodes meanwhile.
    __shared__ int s_il[2], s_iqg[2], s_inqv[2], s_inrows[2];
    __shared__ long long s_irow0[2];
    __shared__ int s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nkb = p.nkb;
    const bool l2 = p.metric == 1;
    volatile int* vabort = &s_abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&accf[i], 1);
            mbar_init(&acce[i], 4);
        }
        s_abort = 0;
        fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(&tbase, TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tbase;
    const uint32_t idesc = tc::idesc_bf16_f32(TM, QG);

    uint32_t load_it = 0;  // producer: k-block loads issued
    uint32_t mma_it = 0;   // MMA issuer: k-blocks consumed
    uint32_t tile_it = 0;  // tiles accumulated (MMA issuer and epilogue count alike)
    const int64_t total_items = p.item_off[p.nlist];

    // Take the next work item from the queue and decode it into slot `slot`
    // (list = the last l with item_off[l] <= g; lists without items are
    // skipped because their item_off equals the next list's).
    auto fetch = [&](int slot) {
        const long long g = atomicAdd(p.work, 1u);
        int l = -1;
        if (g < total_items && !*vabort) {
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
            const int sz = p.list_size[l];
            const int nrs = (sz + p.rs - 1) / p.rs;
            const int qg = w / nrs, rsl = w % nrs;
            s_iqg[slot] = qg;
            s_inqv[slot] = min(QG, p.pair_cnt[l] - qg * QG);
            s_irow0[slot] = p.list_off[l] + static_cast<long long>(rsl) * p.rs;
            s_inrows[slot] = min(p.rs, sz - rsl * p.rs);
        }
        s_il[slot] = l;
    };
    if (threadIdx.x == 64) fetch(0);
    __syncthreads();

    for (int it = 0;; ++it) {
        const int cur = it & 1;
        const int l = s_il[cur];
        if (l < 0) break;
        const int qg = s_iqg[cur], nqv = s_inqv[cur];
        const long long row0 = s_irow0[cur];
        const int nrows = s_inrows[cur];
        const int ntiles = (nrows + TM - 1) / TM;

        // --- gather the group's queries (bf16, swizzled) as the B operand
        const int32_t* grp = p.pairs + p.pair_off[l] + static_cast<int64_t>(qg) * QG;
        for (int i = threadIdx.x; i < QG; i += blockDim.x) {
            const int qid = i < nqv ? grp[i] : -1;
            s_qid[i] = qid;
            if (qid >= 0) {
                const float4 qa = p.qaux[qid];
                const ErrCoef ec = err_coef(qa, l2, p.cK, p.cN);
                s_qn[i] = qa.x;
                s_aq[i] = ec.aq;
                s_bq[i] = ec.bq;
                // A row is a candidate when its bf16 distance minus the error
                // bound is within the query's threshold.
                s_thr[i] = p.thr[qid] + ec.cq;
            } else {
                s_qn[i] = 0.0f;
                s_aq[i] = 0.0f;
                s_bq[i] = 0.0f;
                s_thr[i] = -INFINITY;
            }
        }
        for (int e = threadIdx.x; e < QG * nkb * 8; e += blockDim.x) {
            const int i = e / (nkb * 8), rem = e % (nkb * 8);
            const int kb = rem >> 3, c = rem & 7;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (i < nqv) {
                const int qid = grp[i];
                v = *reinterpret_cast<const uint4*>(p.qb + static_cast<size_t>(qid) * nkb * 64 + kb * 64 + c * 8);
            }
            *reinterpret_cast<uint4*>(sB + kb * KB_BYTES + i * 128 + (((c ^ (i & 7)) & 7) << 4)) = v;
        }
        fence_proxy_async();
        __syncthreads();
        if (threadIdx.x == 64) fetch(cur ^ 1);

        if (warp == 0) {
            // --- producer: k-blocks of the slice's tiles into the stage ring
            if (lane == 0) {
                const int64_t tile0 = row0 / TM;
                for (int t = 0; t < ntiles && !*vabort; ++t) {
                    for (int kb = 0; kb < nkb; ++kb, ++load_it) {
                        const int s = load_it % NS;
                        const uint32_t round = load_it / NS;
                        if (!mbar_wait_bounded(&empty[s], (round & 1u) ^ 1u, p.err)) {
                            s_abort = 1;
                            break;
                        }
                        mbar_expect_tx(&full[s], KB_BYTES);
                        bulk_g2s(sA + static_cast<size_t>(s) * KB_BYTES,
                                 p.abf + ((tile0 + t) * nkb + kb) * static_cast<int64_t>(KB_BYTES), KB_BYTES,
                                 &full[s]);
                    }
                }
            }
        } else if (warp == 1) {
            // --- MMA issuer
            if (lane == 0) {
                for (int t = 0; t < ntiles && !*vabort; ++t, ++tile_it) {
                    const int buf = tile_it & 1;
                    const uint32_t round = tile_it >> 1;
                    if (!mbar_wait_bounded(&acce[buf], (round & 1u) ^ 1u, p.err)) {
                        s_abort = 1;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t dcol = tmem + static_cast<uint32_t>(buf * QG);
                    for (int kb = 0; kb < nkb; ++kb, ++mma_it) {
                        const int s = mma_it % NS;
                        const uint32_t r2 = mma_it / NS;
                        if (!mbar_wait_bounded(&full[s], r2 & 1u, p.err)) {
                            s_abort = 1;
                            break;
                        }
                        tc::fence_after_sync();
                        const uint32_t a0 = smem_u32(sA + static_cast<size_t>(s) * KB_BYTES);
                        const uint32_t b0 = smem_u32(sB + kb * KB_BYTES);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)
                            tc::mma_bf16(dcol, tc::sdesc_sw128(a0 + kk * 32), tc::sdesc_sw128(b0 + kk * 32), idesc,
                                         (kb | kk) != 0 ? 1u : 0u);
                        tc::mma_commit(&empty[s]);
                    }
                    tc::mma_commit(&accf[buf]);
                }
            }
        } else if (warp >= 4) {
            // --- epilogue: thread = row of the tile, 32 queries per TMEM load.
            // Candidates are staged per warp in shared memory (ballot, no
            // atomics) and flushed with one independent atomic per lane.
            const int quad = warp & 3;
            int* wq = s_cq[quad];
            uint64_t* wk = s_ck[quad];
            int wcount = 0;
            auto flush = [&]() {
                __syncwarp();
                for (int i = lane; i < wcount; i += 32) {
                    const int qid = wq[i];
                    const int pos = atomicAdd(&p.cand_cnt[qid], 1);
                    if (pos < p.capq) p.cand[static_cast<int64_t>(qid) * p.capq + pos] = wk[i];
                }
                __syncwarp();
                wcount = 0;
            };
            for (int t = 0; t < ntiles && !*vabort; ++t, ++tile_it) {
                const int buf = tile_it & 1;
                const uint32_t round = tile_it >> 1;
                if (!mbar_wait_bounded(&accf[buf], round & 1u, p.err)) {
                    s_abort = 1;
                    break;
                }
                tc::fence_after_sync();
                const int rs_row = t * TM + quad * 32 + lane;  // row within the slice
                const bool rvalid = rs_row < nrows;
                const int64_t arow = row0 + rs_row;
                float xnv = 0.0f, xnn = 0.0f, xe = 0.0f;
                if (rvalid) {
                    xnv = p.xn[arow];
                    const float2 xa = p.xaux[arow];
                    xnn = xa.x;
                    xe = xa.y;
                }
                const float cx = err_row_const(xnv, l2, p.cN);
                for (int c = 0; c < QG / 32; ++c) {
                    float v[32];
                    tc::tmem_ld32(tmem + (static_cast<uint32_t>(quad * 32) << 16) +
                                      static_cast<uint32_t>(buf * QG + c * 32),
                                  v);
                    if (c * 32 >= nqv) continue;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int qi = c * 32 + j;
                        const float score = l2 ? __fadd_rn(__fadd_rn(xnv, s_qn[qi]), -2.0f * v[j]) : -v[j];
                        const float bound = fmaf(xnn, s_aq[qi], fmaf(xe, s_bq[qi], cx));
                        const bool pass = rvalid && qi < nqv && score - bound <= s_thr[qi];
                        const unsigned m = __ballot_sync(FULL, pass);
                        if (m) {
                            if (wcount + 32 > CB) flush();
                            if (pass) {
                                const int slot = wcount + __popc(m & ((1u << lane) - 1u));
                                wq[slot] = s_qid[qi];
                                wk[slot] = (static_cast<uint64_t>(f2o(score)) << 32) | static_cast<uint32_t>(arow);
                            }
                            wcount += __popc(m);
                        }
                    }
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive_cta(&acce[buf]);
            }
            if (wcount > 0) flush();
        }
        __syncthreads();
        if (*vabort) break;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) tc::tmem_dealloc(tmem, TMEM_COLS);
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

__global__ void __launch_bounds__(256) rerank_kernel(ArenaLayout L, const float* __restrict__ codes,
                                                     const int64_t* __restrict__ ids, const float* __restrict__ xn,
                                                     const float2* __restrict__ xaux, const float4* __restrict__ qaux,
                                                     const float* __restrict__ q, BatchWork w, int qbase, int capq,
                                                     int k, int metric, float cK, float cN, float* __restrict__ D,
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
    const int qi = blockIdx.x;
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
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t key = cq[i];
        const int64_t row = static_cast<int64_t>(key & 0xffffffffu);
        const float sc = o2f(static_cast<uint32_t>(key >> 32));
        const float2 xa = xaux[row];
        const float e = fmaf(xa.x, ec.aq, fmaf(xa.y, ec.bq, err_row_const(xn[row], l2, cN) + ec.cq));
        hi[i] = f2o(sc + e);
        lo[i] = sc - e;
    }
    __syncthreads();
    float U = INFINITY;
    if (n > k) {
        int need;
        U = o2f(cta_radix_select(hi, n, k, &need, hist, sh));
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (lo[i] <= U) {
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
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
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
static void err_consts(int d, float* cK, float* cN) {
    const int K = (d + 63) / 64 * 64;
    const double u = 1.0 / 16777216.0, inflate = 1.0 + 1.0 / 128.0;
    *cK = static_cast<float>((K + 8) * u * inflate);
    *cN = static_cast<float>((3.0 * d + 16) * u * inflate);
}

cudaError_t launch_fill_f32(float* p, int64_t n, float v, cudaStream_t s) {
    fill_f32_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t launch_prep_queries(const float* q, int nq, int d, void* qb, float4* qaux, cudaStream_t s) {
    const int nkb = (d + 63) / 64;
    prep_queries_kernel<<<nq, 128, 0, s>>>(q, nq, d, nkb, static_cast<__nv_bfloat16*>(qb), qaux);
    return cudaGetLastError();
}

cudaError_t launch_row_aux(const ArenaLayout& L, const float* codes, int64_t rows, float2* aux, cudaStream_t s) {
    row_aux_kernel<<<grid_for(rows * 32, 256), 256, 0, s>>>(L, codes, rows, aux);
    return cudaGetLastError();
}

cudaError_t launch_invert_probes(const int64_t* probes, int nq, int nprobe, int nlist, const int32_t* list_size,
                                 int rs, const BatchWork& w, cudaStream_t s) {
    const int64_t n = static_cast<int64_t>(nq) * nprobe;
    cudaError_t e;
    if ((e = cudaMemsetAsync(w.pair_cnt, 0, nlist * sizeof(int32_t), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.pair_fill, 0, nlist * sizeof(int32_t), s)) != cudaSuccess) return e;
    probe_hist_kernel<<<grid_for(n, 256), 256, 0, s>>>(probes, n, w.pair_cnt);
    scan_kernel<<<1, 1024, 0, s>>>(w.pair_cnt, nlist, w.pair_off);
    probe_fill_kernel<<<grid_for(n, 256), 256, 0, s>>>(probes, nq, nprobe, w.pair_off, w.pair_fill, w.pairs);
    item_count_kernel<<<grid_for(nlist, 256), 256, 0, s>>>(w.pair_cnt, list_size, nlist, rs, w.item_cnt);
    scan_kernel<<<1, 1024, 0, s>>>(w.item_cnt, nlist, w.item_off);
    return cudaGetLastError();
}

cudaError_t launch_batched_scan(const BatchedLaunch& b, const BatchWork& w, int* err, cudaStream_t s) {
    BatchedParams p;
    p.abf = static_cast<const unsigned char*>(b.abf);
    p.list_off = b.list_off;
    p.list_size = b.list_size;
    p.item_off = w.item_off;
    p.pair_off = w.pair_off;
    p.pairs = w.pairs;
    p.pair_cnt = w.pair_cnt;
    p.xn = b.xn;
    p.xaux = b.xaux;
    p.qb = static_cast<const __nv_bfloat16*>(b.qb);
    p.qaux = b.qaux;
    p.thr = b.thr;
    p.cand = w.cand;
    p.cand_cnt = w.cand_cnt;
    p.work = w.work;
    p.err = err;
    p.nlist = b.nlist;
    p.nkb = (b.d + 63) / 64;
    p.rs = b.rs;
    p.capq = b.capq;
    p.metric = b.metric;
    err_consts(b.d, &p.cK, &p.cN);
    const size_t smem = 1024 + static_cast<size_t>(p.nkb) * KB_BYTES + static_cast<size_t>(NS) * KB_BYTES;
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = cudaMemsetAsync(w.work, 0, sizeof(unsigned int), s)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(batched_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem))) != cudaSuccess)
        return e;
    batched_scan_kernel<<<b.nsm, 256, smem, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_rerank(const ArenaLayout& L, const float* codes, const int64_t* ids, const float* xn,
                          const float2* xaux, const float4* qaux, const float* q, int nq, const BatchWork& w, int qbase,
                          int capq, int k, int metric, float* D, int64_t* I, cudaStream_t s) {
    const size_t smem = static_cast<size_t>(RERANK_MAX) * 8 + static_cast<size_t>(L.row_pitch) * 4 +
                        static_cast<size_t>(capq) * 8;
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(rerank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    float cK, cN;
    err_consts(L.d, &cK, &cN);
    rerank_kernel<<<nq, 256, smem, s>>>(L, codes, ids, xn, xaux, qaux, q, w, qbase, capq, k, metric, cK, cN, D, I);
    return cudaGetLastError();
}

}  // namespace hy
