// CPU restatement of Harmony's IVF query path — the ORACLE.
//
// TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg use this library as the checker.  The product library
// (harmonyclient_b200/libhy.so) never links, loads or calls it, and has no CPU
// fallback.
//
// Each function restates one step of the reference (paths relative to the
// reference repository) in plain, sequential C++ written for this project.
// Float sums run left to right in single precision, as the reference's scalar
// loops are written (src/utils.h:480-519); the reference's Release build
// vectorises them, so on non-integer data the two can differ in the last ulp.
// The restatement is pinned against the reference itself (oracle/_ref, built
// from the reference sources) by tests/test_oracle_pinned.py and the golden
// fixtures under tests/golden/.
//
// Storage used throughout: inverted lists as CSR — offsets[nlist+1] (rows),
// ids[nb] (int64 source row), codes[nb*d] row-major in list order.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <vector>

typedef int64_t idx_t;
enum { OC_METRIC_IP = 0, OC_METRIC_L2 = 1 };

extern "C" {

// Squared L2 distance, sequential float sum (src/utils.h:480-487).
float oc_l2(const float* a, const float* b, size_t d) {
    float s = 0.0f;
    for (size_t i = 0; i < d; ++i) {
        float t = a[i] - b[i];
        s += t * t;
    }
    return s;
}

// Inner product, sequential float sum (src/utils.h:512-519).
float oc_ip(const float* a, const float* b, size_t d) {
    float s = 0.0f;
    for (size_t i = 0; i < d; ++i) s += a[i] * b[i];
    return s;
}

}  // extern "C"

namespace {

// "a is worse than b" for the metric: larger for L2, smaller for IP.
inline bool worse(int metric, float a, float b) { return metric == OC_METRIC_L2 ? a > b : a < b; }

// heap_init (src/heap.hpp:13-25): L2 heaps start at FLT_MAX, IP at lowest.
void heap_init(int metric, size_t k, float* v, idx_t* id) {
    for (size_t i = 0; i < k; ++i) {
        v[i] = metric == OC_METRIC_L2 ? FLT_MAX : -FLT_MAX;
        id[i] = -1;
    }
}

// heap_replace_top (src/heap.hpp:35-71): a 1-based binary heap whose root is
// the worst kept entry; the new value sinks while a child is not worse than it.
void heap_replace_top(int metric, size_t k, float* v, idx_t* id, float val, idx_t vid) {
    float* hv = v - 1;
    idx_t* hi = id - 1;
    size_t i = 1;
    for (;;) {
        size_t l = 2 * i, r = l + 1;
        if (l > k) break;
        size_t c;
        if (r == k + 1 || worse(metric, hv[l], hv[r]))
            c = l;
        else
            c = r;
        if (worse(metric, val, hv[c])) break;
        hv[i] = hv[c];
        hi[i] = hi[c];
        i = c;
    }
    hv[i] = val;
    hi[i] = vid;
}

// heap_sort (src/heap.hpp:73-82): repeatedly move the root to the end, so the
// result is best-first (ascending L2, descending IP).
void heap_sort(int metric, size_t k, float* v, idx_t* id) {
    for (int64_t i = static_cast<int64_t>(k) - 1; i >= 0; --i) {
        float val = v[i];
        idx_t vid = id[i];
        v[i] = v[0];
        id[i] = id[0];
        heap_replace_top(metric, static_cast<size_t>(i), v, id, val, vid);
    }
}

// The strict admission test every reference scan loop uses before
// heap_replace_top (src/IVFScan.hpp:122,131,267).
inline bool admits(int metric, float dis, float top) { return metric == OC_METRIC_L2 ? dis < top : dis > top; }

inline float dist(int metric, const float* a, const float* b, size_t d) {
    return metric == OC_METRIC_L2 ? oc_l2(a, b, d) : oc_ip(a, b, d);
}

}  // namespace

extern "C" {

// Top-k of a value stream through the reference heap discipline.
int oc_heap_topk(int metric, size_t n, const float* vals, const idx_t* ids, size_t k, float* out_v, idx_t* out_i) {
    heap_init(metric, k, out_v, out_i);
    for (size_t i = 0; i < n; ++i)
        if (admits(metric, vals[i], out_v[0])) heap_replace_top(metric, k, out_v, out_i, vals[i], ids[i]);
    heap_sort(metric, k, out_v, out_i);
    return 0;
}

// Coarse quantisation (src/Index.cpp:967-995 with IVFScan::lite_scan_codes,
// src/IVFScan.hpp:108-138): per query, the nprobe best centroids, best first.
int oc_probes(size_t nq, const float* q, size_t nlist, const float* cent, size_t d, int metric, size_t nprobe,
              idx_t* probes, float* pdist) {
    if (nprobe > nlist) nprobe = nlist;
    std::vector<float> hv(nprobe);
    std::vector<idx_t> hi(nprobe);
#pragma omp parallel for firstprivate(hv, hi) schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(nq); ++i) {
        heap_init(metric, nprobe, hv.data(), hi.data());
        for (size_t c = 0; c < nlist; ++c) {
            float s = dist(metric, q + i * d, cent + c * d, d);
            if (admits(metric, s, hv[0])) heap_replace_top(metric, nprobe, hv.data(), hi.data(), s, (idx_t)c);
        }
        heap_sort(metric, nprobe, hv.data(), hi.data());
        std::copy(hi.begin(), hi.end(), probes + i * nprobe);
        if (pdist) std::copy(hv.begin(), hv.end(), pdist + i * nprobe);
    }
    return 0;
}

// Nearest centroid per row (src/Index.cpp:567-579 via lite_scan_codes with
// k=1): the first strictly better centroid wins ties.
int oc_assign(size_t n, const float* x, size_t nlist, const float* cent, size_t d, int metric, idx_t* labels,
              float* dis) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
        float best = metric == OC_METRIC_L2 ? FLT_MAX : -FLT_MAX;
        idx_t bl = -1;
        for (size_t c = 0; c < nlist; ++c) {
            float s = dist(metric, x + i * d, cent + c * d, d);
            if (admits(metric, s, best)) {
                best = s;
                bl = (idx_t)c;
            }
        }
        labels[i] = bl;
        dis[i] = best;
    }
    return 0;
}

// Index::add list construction (src/Index.cpp:624-671): list sizes, then rows
// placed in order of their distance to the centroid (ascending for L2,
// descending for IP).  The reference uses an unstable std::sort; ties are
// broken here by source row so the order is deterministic.
// Outputs: offsets[nlist+1]; order[n] = source row of each arena slot.
int oc_build_lists(size_t n, size_t nlist, int metric, const idx_t* labels, const float* dis, idx_t* offsets,
                   idx_t* order) {
    std::vector<idx_t> cnt(nlist, 0);
    for (size_t i = 0; i < n; ++i) cnt[labels[i]]++;
    offsets[0] = 0;
    for (size_t l = 0; l < nlist; ++l) offsets[l + 1] = offsets[l] + cnt[l];
    std::vector<idx_t> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](idx_t a, idx_t b) {
        if (dis[a] != dis[b]) return metric == OC_METRIC_L2 ? dis[a] < dis[b] : dis[a] > dis[b];
        return false;
    });
    std::vector<idx_t> fill(offsets, offsets + nlist);
    for (size_t oi = 0; oi < n; ++oi) {
        idx_t i = ord[oi];
        order[fill[labels[i]]++] = i;
    }
    return 0;
}

// The plain exact IVF-flat scan with caller-given probe lists: for each
// probed list in order, each row in list order, full-d distance, strict
// admission against the heap top, then heap_sort (src/Index.cpp:1450-1547,
// src/IVFScan.hpp:240-288; IP branch src/Index.cpp:1509-1546 without the
// optional OPT_TRIANGLE window).
int oc_scan_probes(size_t nq, const float* q, size_t d, const idx_t* offsets, const idx_t* ids, const float* codes,
                   int metric, size_t nprobe, const idx_t* probes, size_t k, float* D, idx_t* I) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < static_cast<int64_t>(nq); ++i) {
        float* v = D + i * k;
        idx_t* id = I + i * k;
        heap_init(metric, k, v, id);
        const float* qi = q + i * d;
        for (size_t j = 0; j < nprobe; ++j) {
            idx_t l = probes[i * nprobe + j];
            if (l < 0) continue;
            for (idx_t r = offsets[l]; r < offsets[l + 1]; ++r) {
                float s = dist(metric, qi, codes + r * d, d);
                if (admits(metric, s, v[0])) heap_replace_top(metric, k, v, id, s, ids[r]);
            }
        }
        heap_sort(metric, k, v, id);
    }
    return 0;
}

// Warm-up pruning thresholds (src/Index.cpp:999-1051 and 1300-1303): scan the
// first min(warmup_list, nprobe) probed lists, at most warmup_list_size rows
// of each, into a fresh heap; heapTop = the heap's root (its k-th best, or
// FLT_MAX while fewer than k rows were seen).  L2 only, as in the reference.
int oc_warmup_tops(size_t nq, const float* q, size_t d, const idx_t* offsets, const float* codes, size_t nprobe,
                   const idx_t* probes, size_t k, size_t warmup_list, size_t warmup_list_size, float* tops) {
    size_t wl = std::min(warmup_list, nprobe);
    std::vector<float> hv(k);
    std::vector<idx_t> hi(k);
#pragma omp parallel for firstprivate(hv, hi) schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(nq); ++i) {
        heap_init(OC_METRIC_L2, k, hv.data(), hi.data());
        for (size_t j = 0; j < wl; ++j) {
            idx_t l = probes[i * nprobe + j];
            idx_t sz = offsets[l + 1] - offsets[l];
            idx_t m = std::min<idx_t>(sz, (idx_t)warmup_list_size);
            for (idx_t r = offsets[l]; r < offsets[l] + m; ++r) {
                float s = oc_l2(q + i * d, codes + r * d, d);
                if (s < hv[0]) heap_replace_top(OC_METRIC_L2, k, hv.data(), hi.data(), s, r);
            }
        }
        tops[i] = hv[0];
    }
    return 0;
}

// Partial-distance pruning scan (BaseWorker::single_thread_search_simple with
// cut, src/node.cpp:634-657): d is split into nblocks chunks of d/nblocks dims,
// the last taking the remainder; after each chunk but the last, a partial sum
// above the query's threshold prunes the row.  Survivors go through the same
// strict heap admission.  Returns the number of (row, chunk) evaluations
// skipped through *skipped when non-null.
int oc_scan_prune(size_t nq, const float* q, size_t d, const idx_t* offsets, const idx_t* ids, const float* codes,
                  size_t nprobe, const idx_t* probes, const float* tops, size_t k, size_t nblocks, float* D, idx_t* I,
                  int64_t* skipped) {
    size_t cd = d / nblocks;
    int64_t skip_total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : skip_total)
    for (int64_t i = 0; i < static_cast<int64_t>(nq); ++i) {
        float* v = D + i * k;
        idx_t* id = I + i * k;
        heap_init(OC_METRIC_L2, k, v, id);
        const float* qi = q + i * d;
        for (size_t j = 0; j < nprobe; ++j) {
            idx_t l = probes[i * nprobe + j];
            if (l < 0) continue;
            for (idx_t r = offsets[l]; r < offsets[l + 1]; ++r) {
                const float* x = codes + r * d;
                float s = 0.0f;
                for (size_t b = 0; b < nblocks; ++b) {
                    size_t w = (b == nblocks - 1) ? d - b * cd : cd;
                    s += oc_l2(qi + b * cd, x + b * cd, w);
                    if (b + 1 < nblocks && s > tops[i]) {
                        s = INFINITY;
                        skip_total += static_cast<int64_t>(nblocks - b - 1);
                        break;
                    }
                }
                if (s < v[0]) heap_replace_top(OC_METRIC_L2, k, v, id, s, ids[r]);
            }
        }
        heap_sort(OC_METRIC_L2, k, v, id);
    }
    if (skipped) *skipped = skip_total;
    return 0;
}

// k-means training (Clustering::train, src/Clustering.cpp:14-152, with the
// parameters Index::train passes, src/Index.cpp:386-394):
//  - subsample to nlist*max_points_per_centroid rows when n exceeds it, by a
//    std::shuffle of 0..n-1 under std::default_random_engine(seed);
//  - initial centroids = the sample rows at the first nlist entries of a
//    second shuffle (same engine and seed) of 0..n_sample-1;
//  - niter Lloyd steps: nearest centroid (L2: first strict minimum; IP: first
//    strict maximum over L2-normalised rows), then each non-empty centroid
//    becomes the mean of its RAW rows; empty ones keep their value;
//  - IP: centroids are L2-normalised at the end (src/Index.cpp:408-419).
// fp64_accum selects double accumulation of the sums (as the GPU does);
// otherwise sums are float in row order (the reference with one thread).
int oc_kmeans(size_t n, const float* x, size_t d, size_t nlist, int niter, int seed, size_t max_points_per_centroid,
              int metric, int fp64_accum, float* centroids) {
    std::vector<float> sample;
    const float* xs = x;
    size_t ns = n;
    size_t maxs = nlist * max_points_per_centroid;
    if (n > maxs) {
        std::vector<size_t> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        std::shuffle(idx.begin(), idx.end(), std::default_random_engine(seed));
        sample.resize(maxs * d);
        for (size_t i = 0; i < maxs; ++i) std::memcpy(&sample[i * d], x + idx[i] * d, d * sizeof(float));
        xs = sample.data();
        ns = maxs;
    }
    {
        std::vector<size_t> idx(ns);
        std::iota(idx.begin(), idx.end(), 0);
        std::shuffle(idx.begin(), idx.end(), std::default_random_engine(seed));
        for (size_t c = 0; c < nlist; ++c) std::memcpy(centroids + c * d, xs + idx[c] * d, d * sizeof(float));
    }
    std::vector<float> xn;
    if (metric == OC_METRIC_IP) {
        xn.assign(xs, xs + ns * d);
        for (size_t i = 0; i < ns; ++i) {
            float s = 0.0f;
            for (size_t j = 0; j < d; ++j) s += xn[i * d + j] * xn[i * d + j];
            float nr = std::sqrt(s);
            if (nr > 0.0f)
                for (size_t j = 0; j < d; ++j) xn[i * d + j] /= nr;
        }
    }
    std::vector<idx_t> lab(ns);
    std::vector<double> accd;
    std::vector<float> accf;
    std::vector<size_t> cnt(nlist);
    for (int it = 0; it < niter; ++it) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < static_cast<int64_t>(ns); ++i) {
            const float* r = metric == OC_METRIC_IP ? &xn[i * d] : xs + i * d;
            float best = metric == OC_METRIC_L2 ? FLT_MAX : -FLT_MAX;
            idx_t bl = 0;
            for (size_t c = 0; c < nlist; ++c) {
                float s = dist(metric, r, centroids + c * d, d);
                if (admits(metric, s, best)) {
                    best = s;
                    bl = (idx_t)c;
                }
            }
            lab[i] = bl;
        }
        std::fill(cnt.begin(), cnt.end(), 0);
        if (fp64_accum) {
            accd.assign(nlist * d, 0.0);
            for (size_t i = 0; i < ns; ++i) {
                cnt[lab[i]]++;
                for (size_t j = 0; j < d; ++j) accd[lab[i] * d + j] += xs[i * d + j];
            }
            for (size_t c = 0; c < nlist; ++c)
                if (cnt[c] > 0)
                    for (size_t j = 0; j < d; ++j)
                        centroids[c * d + j] = static_cast<float>(accd[c * d + j] / static_cast<double>(cnt[c]));
        } else {
            accf.assign(nlist * d, 0.0f);
            for (size_t i = 0; i < ns; ++i) {
                cnt[lab[i]]++;
                for (size_t j = 0; j < d; ++j) accf[lab[i] * d + j] += xs[i * d + j];
            }
            for (size_t c = 0; c < nlist; ++c)
                if (cnt[c] > 0)
                    for (size_t j = 0; j < d; ++j) centroids[c * d + j] = accf[c * d + j] / static_cast<float>(cnt[c]);
        }
    }
    if (metric == OC_METRIC_IP) {
        for (size_t c = 0; c < nlist; ++c) {
            float s = oc_ip(centroids + c * d, centroids + c * d, d);
            if (s != 0.0f)
                for (size_t j = 0; j < d; ++j) centroids[c * d + j] /= std::sqrt(s);
        }
    }
    return 0;
}

// Exact brute force in double precision: the recall truth (the reference uses
// faiss IndexIVFFlat at nprobe=nlist, src/query.cpp:856-868, which is exact
// search; this oracle computes it in FP64).  Ties broken by lower row id.
int oc_bruteforce_f64(size_t nb, const float* x, size_t nq, const float* q, size_t d, int metric, size_t k, double* D,
                      idx_t* I) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < static_cast<int64_t>(nq); ++i) {
        std::vector<std::pair<double, idx_t>> all(nb);
        for (size_t r = 0; r < nb; ++r) {
            double s = 0.0;
            for (size_t j = 0; j < d; ++j) {
                double a = q[i * d + j], b = x[r * d + j];
                s += metric == OC_METRIC_L2 ? (a - b) * (a - b) : a * b;
            }
            all[r] = {metric == OC_METRIC_L2 ? s : -s, (idx_t)r};
        }
        size_t kk = std::min(k, nb);
        std::partial_sort(all.begin(), all.begin() + kk, all.end());
        for (size_t j = 0; j < k; ++j) {
            if (j < kk) {
                D[i * k + j] = metric == OC_METRIC_L2 ? all[j].first : -all[j].first;
                I[i * k + j] = all[j].second;
            } else {
                D[i * k + j] = metric == OC_METRIC_L2 ? INFINITY : -INFINITY;
                I[i * k + j] = -1;
            }
        }
    }
    return 0;
}

}  // extern "C"
