// C-ABI of the B200 IVF engine: handle lifecycle, training, list
// construction, search orchestration, list access and the reference's .index
// file format.  Declarations and contracts are in include/hy.h.
//
// Everything on the data path runs on the GPU through the kernels in
// hy_kernels.cu; host code here only validates arguments, sizes buffers,
// computes the seeded sampling permutation (std::shuffle with
// std::default_random_engine, as the reference's Clustering does) and moves
// data between host and device.  There is no CPU search path.
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/hy.h"
#include "hy_batched.cuh"
#include "hy_lists.cuh"
#include "hy_kernels.cuh"
#include "hy_mlp.cuh"

using hy::ArenaLayout;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

struct Status {
    int code = HY_OK;
    std::string msg;
};

#define HY_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? HY_ERR_OOM : HY_ERR_CUDA,                    \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                           \
        }                                                                                              \
    } while (0)

#define HY_CHECK(cond, code, msg) \
    do {                          \
        if (!(cond)) return fail(code, msg); \
    } while (0)

#define HY_RET(call)              \
    do {                          \
        int rc_ = (call);         \
        if (rc_ != HY_OK) return rc_; \
    } while (0)

// A grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    int ensure(size_t n) {
        if (n <= bytes) return HY_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        size_t want = std::max<size_t>(n, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(HY_ERR_OOM, std::string("cudaMalloc(") + std::to_string(want) + "): " + cudaGetErrorString(e));
        }
        bytes = want;
        return HY_OK;
    }
    // ensure(n), and zero the bytes when they were just allocated.
    int ensure_zeroed(size_t n) {
        const bool fresh = n > bytes;
        int rc = ensure(n);
        if (rc == HY_OK && fresh && cudaMemset(p, 0, bytes) != cudaSuccess)
            return fail(HY_ERR_CUDA, "cudaMemset of a new buffer failed");
        return rc;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

ArenaLayout make_layout(int d, int nb) {
    ArenaLayout L;
    L.d = d;
    L.nb = nb;
    const int cd = d / nb;
    for (int b = 0; b < nb; ++b) L.bstart[b] = b * cd;
    L.bstart[nb] = d;
    L.boff[0] = 0;
    L.max_pitch = 0;
    for (int b = 0; b < nb; ++b) {
        const int w = L.bstart[b + 1] - L.bstart[b];
        L.pitch[b] = (w + hy::PITCH_ALIGN - 1) / hy::PITCH_ALIGN * hy::PITCH_ALIGN;
        L.boff[b + 1] = L.boff[b] + L.pitch[b];
        L.max_pitch = std::max(L.max_pitch, L.pitch[b]);
    }
    L.row_pitch = L.boff[nb];
    return L;
}

}  // namespace

// Device status of a host-pointer call, read back in one pinned block.
struct HostStatus {
    int err = 0;
    unsigned long long counters[4] = {0, 0, 0, 0};  // scan counters (block copies, blocks unpruned, block sums, sums unpruned)
    unsigned long long learned_total = 0;     // sum of the learned nprobes
    unsigned long long fallback = 0;  // queries answered by the device fallback
};

struct hy_index {
    std::mutex mu;
    int device = 0;
    size_t d = 0, nlist = 0, nprobe = 0;
    int metric = HY_METRIC_L2;
    int opt_level = 0;
    size_t sub_k = 0, sub_nlist = 1, sub_nprobe = 1;
    size_t dim_blocks = 4;
    ArenaLayout L;
    bool trained = false;
    size_t ntotal = 0;
    size_t arena_rows = 0;
    size_t warmup_list = 0, warmup_list_size = 0;

    std::vector<float> h_cent;
    std::vector<int64_t> h_list_off;  // nlist+1, arena rows (tile aligned)
    std::vector<int32_t> h_list_size;

    DevBuf cent, list_off, list_size, ids, codes, norms;
    // workspace
    DevBuf w_q, w_scores, w_probes, w_thr, w_gthr, w_parts, w_D, w_I, w_f, w_counters, w_err;
    DevBuf w_x, w_lab, w_dist, w_keys, w_keys2, w_vals, w_vals2, w_sort, w_start, w_sums, w_cnt, w_rows, w_xn;

    cudaStream_t stream = nullptr;
    // Timing events (0-4: phases; 6-9: the batched scan launches).  A search
    // captured in a graph records its own set: an event recorded during a
    // capture cannot be waited on outside the graph.
    cudaEvent_t ev_direct[10] = {};
    cudaEvent_t ev_graph[10] = {};
    cudaEvent_t* ev = ev_direct;
    int kev = 0;              // batched scan launches timed by ev[6..9]
    size_t list_lo = 0, list_hi = SIZE_MAX;  // lists this index holds (hy_index_set_list_range)
    size_t learned_rows = SIZE_MAX;  // the learned cut applies to batch rows below this
    DevBuf w_jrows;                  // judged rows of a learned batch
    const int32_t* q_nprobe = nullptr;  // per-query nprobe (device) during a search_nprobes call
    DevBuf w_np;
    // CUDA graph of the device-pointer search (graph mode): the captured
    // launch sequence and the call it was captured for.
    uint64_t epoch = 0;  // bumped by every call that changes what a search does
    bool graph_on = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    struct GraphKey {
        uint64_t epoch;
        size_t n, k, nprobe;
        const void *dq, *dD, *dI, *np;
        cudaStream_t s;
        size_t learned_rows;
        int learned;
        bool operator==(const GraphKey& o) const {
            return epoch == o.epoch && n == o.n && k == o.k && nprobe == o.nprobe && dq == o.dq && dD == o.dD &&
                   dI == o.dI && np == o.np && s == o.s && learned_rows == o.learned_rows && learned == o.learned;
        }
    } gkey{};
    uint64_t graph_kernels = 0;
    int graph_kev = 0;
    cudaEvent_t gev[2] = {};
    bool times_pending = false;  // a device-API search recorded events not yet read
    HostStatus* hstat = nullptr;  // pinned status block of host-pointer calls (finish_host_call)
    int64_t* hjudge = nullptr;    // pinned results of the learned judge's rows
    size_t hjudge_cap = 0;
    hy_search_stats_t stats = {};
    uint64_t launches = 0;  // kernels launched since the last stats snapshot

    // plain form: query-major or list-major scan (hy_index_set_plain_scan)
    int plain_scan = HY_PLAIN_AUTO;
    bool lm_last = false;  // the last plain search ran the list-major scan
    // batched tensor-core forms (bf16, e4m3)
    int form = HY_FORM_PLAIN;
    size_t capq = 8192;       // candidate slots per query
    size_t oversample = 4;    // e4m3 form: exact re-rank of at most oversample * k candidates
    size_t row_slice = 2048;  // rows per work item
    int group_size = 0;       // queries per group of the search passes (0: per pass, by queries per list)
    double learned_mean = 0;  // the probe model's held-out mean nprobe (0: unknown)
    int nsm = 0;
    DevBuf abf;               // bf16 tensor-core image of the arena
    DevBuf xaux;              // per arena row {|x~|, |x - x~|}
    DevBuf taux;              // per 128-row tile, maxima of xaux
    DevBuf txn;               // per 128-row tile, the largest squared norm
    bool abf_valid = false;
    DevBuf b_cert;            // the bf16 image's exactness certificate {integral, max row norm}
    float arena_maxxn = -1.0f;  // its largest row squared norm when integral (<= 256), else -1
    DevBuf b_qx;              // per-query exact-distance flags
    DevBuf a8, x8aux, t8aux;  // the same for the e4m3 image
    DevBuf lscale, tscale, tmax;  // e4m3 per-list and per-tile scales, tile maxima
    bool a8_valid = false;
    DevBuf b_qs;              // e4m3 per-query scales
    DevBuf b_big;             // queries re-ranked by the CTA kernel
    DevBuf b_qb, b_qn, b_thr, b_pcnt, b_pfill, b_poff, b_pairs, b_icnt, b_ioff, b_work, b_cand, b_ccnt, b_ovf, b_items;
    DevBuf b_done;            // the probe inversion's ticket (zero between launches)
    DevBuf b_fq, b_fpr, b_fD, b_fI, b_fcnt, b_fbtot;  // device-side exact fallback
    // coarse quantiser on the tensor cores (bf16 form): the centroids as a
    // one-list index (image, row aux, tile aux, norms, list offsets/sizes)
    // and the work of one launch
    int coarse_mode = HY_COARSE_TENSOR;
    bool cimg_valid = false;
    // Inner product with OPT_TRIANGLE: per arena row its inner product with
    // its list's centroid and per 32-row tile {max, min} (built on first use).
    DevBuf c2c, c2c_tile;
    bool c2c_valid = false;
    DevBuf c_img, c_aux, c_taux, c_norm, c_off, c_size;
    DevBuf c_pcnt, c_poff, c_pairs, c_ioff, c_items, c_work, c_cand, c_ccnt;

    // learned probe predictor
    bool model_ready = false;
    int learned = 0;
    float judge_fraction = 0.01f, judge_recall = 0.95f;
    float margin = 0.0f;
    int model_P = 0;
    DevBuf m_params, m_mu, m_sd, m_X, m_y, m_work, m_pscore, m_total;
    DevBuf m_wimg;  // the weights' tensor-core operand image (mlp_pack)
    DevBuf t_X, t_t, t_Xb, t_tb, t_dy, t_loss, t_grads, t_am, t_av, t_perm, t_rows, t_D, t_I;
};

namespace {

// Timing events are recorded as external event nodes when the stream is
// being captured, so a replayed graph records them too.
inline cudaError_t ev_record(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    const cudaError_t ce = cudaStreamIsCapturing(s, &st);
    if (ce != cudaSuccess) return ce;
    return st == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal)
                                               : cudaEventRecord(e, s);
}

int set_device(hy_index* h) {
    HY_CUDA(cudaSetDevice(h->device));
    return HY_OK;
}

// Bytes of the coarse score scratch per query chunk.
constexpr size_t SCORE_BUDGET = size_t(512) << 20;

size_t query_chunk(size_t nlist, size_t n) {
    size_t qc = SCORE_BUDGET / (nlist * sizeof(float));
    qc = std::max<size_t>(qc, 64);
    qc = std::min<size_t>(qc, 65536);
    return std::min(qc, n);
}

// Nearest centroid of each of n device rows (x), chunked: labels, scores.
int assign_rows(hy_index* h, const float* x, size_t n, int64_t* labels, float* score, cudaStream_t s) {
    const size_t rc = query_chunk(h->nlist, n);
    HY_RET(h->w_scores.ensure(rc * h->nlist * sizeof(float)));
    for (size_t r0 = 0; r0 < n; r0 += rc) {
        const size_t m = std::min(rc, n - r0);
        HY_CUDA(hy::launch_coarse_scores(x + r0 * h->d, (int)m, h->cent.as<float>(), (int)h->nlist, (int)h->d,
                                         h->metric, h->w_scores.as<float>(), s));
        HY_CUDA(hy::launch_argmin(h->w_scores.as<float>(), (int)m, (int)h->nlist, labels + r0, score ? score + r0 : nullptr,
                                  s));
    }
    return HY_OK;
}

// k-means on a device sample xs (ns rows): centroids initialised from host
// sample indices; FP64 sums (Clustering::update_centroids,
// src/Clustering.cpp:93-152).
int kmeans_device(hy_index* h, const float* xs, size_t ns, const std::vector<int64_t>& init_rows, int niter,
                  cudaStream_t s) {
    const size_t d = h->d, nlist = h->nlist;
    HY_RET(h->w_rows.ensure(nlist * sizeof(int64_t)));
    HY_CUDA(cudaMemcpyAsync(h->w_rows.p, init_rows.data(), nlist * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    HY_RET(h->cent.ensure(nlist * d * sizeof(float)));
    HY_CUDA(hy::launch_gather_rows(xs, h->w_rows.as<int64_t>(), (int64_t)nlist, (int)d, h->cent.as<float>(), s));
    const float* assign_src = xs;
    if (h->metric == HY_METRIC_IP) {
        HY_RET(h->w_xn.ensure(ns * d * sizeof(float)));
        HY_CUDA(hy::launch_normalize_rows(xs, (int64_t)ns, (int)d, h->w_xn.as<float>(), s));
        assign_src = h->w_xn.as<float>();
    }
    HY_RET(h->w_lab.ensure(ns * sizeof(int64_t)));
    HY_RET(h->w_sums.ensure(nlist * d * sizeof(double)));
    HY_RET(h->w_cnt.ensure(nlist * sizeof(unsigned long long)));
    for (int it = 0; it < niter; ++it) {
        HY_RET(assign_rows(h, assign_src, ns, h->w_lab.as<int64_t>(), nullptr, s));
        HY_CUDA(cudaMemsetAsync(h->w_sums.p, 0, nlist * d * sizeof(double), s));
        HY_CUDA(cudaMemsetAsync(h->w_cnt.p, 0, nlist * sizeof(unsigned long long), s));
        HY_CUDA(hy::launch_kmeans_accumulate(xs, h->w_lab.as<int64_t>(), (int64_t)ns, (int)d, h->w_sums.as<double>(),
                                             h->w_cnt.as<unsigned long long>(), s));
        HY_CUDA(hy::launch_kmeans_update(h->w_sums.as<double>(), h->w_cnt.as<unsigned long long>(), (int)nlist, (int)d,
                                         h->cent.as<float>(), s));
    }
    if (h->metric == HY_METRIC_IP) HY_CUDA(hy::launch_normalize_centroids(h->cent.as<float>(), (int)nlist, (int)d, s));
    h->h_cent.resize(nlist * d);
    HY_CUDA(cudaMemcpyAsync(h->h_cent.data(), h->cent.p, nlist * d * sizeof(float), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaStreamSynchronize(s));
    h->trained = true;
    h->cimg_valid = false;
    return HY_OK;
}

// The reference's sampling: keep everything when n <= nlist * 256, else the
// first nlist*256 entries of a shuffle of 0..n-1 (src/Clustering.cpp:48-68);
// initial centroids are the first nlist entries of a second shuffle of the
// sample (src/Clustering.cpp:72-89).  Both shuffles use
// std::default_random_engine(6666) (src/Index.cpp:392).
void sampling_plan(size_t n, size_t nlist, std::vector<int64_t>* sample, std::vector<int64_t>* init, size_t* ns) {
    const size_t maxs = nlist * 256;
    const int seed = 6666;
    sample->clear();
    *ns = n;
    if (n > maxs) {
        std::vector<size_t> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        std::shuffle(idx.begin(), idx.end(), std::default_random_engine(seed));
        sample->assign(idx.begin(), idx.begin() + maxs);
        *ns = maxs;
    }
    std::vector<size_t> idx2(*ns);
    std::iota(idx2.begin(), idx2.end(), 0);
    std::shuffle(idx2.begin(), idx2.end(), std::default_random_engine(seed));
    init->assign(idx2.begin(), idx2.begin() + nlist);
}

int train_impl(hy_index* h, size_t n, const float* x, bool x_on_device, int lite, cudaStream_t s) {
    HY_CHECK(n >= h->nlist, HY_ERR_ARG, "train: need at least nlist training rows");
    std::vector<int64_t> sample, init;
    size_t ns = 0;
    sampling_plan(n, h->nlist, &sample, &init, &ns);
    const size_t d = h->d;
    HY_RET(h->w_x.ensure(ns * d * sizeof(float)));
    float* xs = h->w_x.as<float>();
    if (x_on_device) {
        if (sample.empty()) {
            HY_CUDA(cudaMemcpyAsync(xs, x, ns * d * sizeof(float), cudaMemcpyDeviceToDevice, s));
        } else {
            HY_RET(h->w_keys.ensure(ns * sizeof(int64_t)));
            HY_CUDA(cudaMemcpyAsync(h->w_keys.p, sample.data(), ns * sizeof(int64_t), cudaMemcpyHostToDevice, s));
            HY_CUDA(hy::launch_gather_rows(x, h->w_keys.as<int64_t>(), (int64_t)ns, (int)d, xs, s));
        }
    } else {
        if (sample.empty()) {
            HY_CUDA(cudaMemcpyAsync(xs, x, ns * d * sizeof(float), cudaMemcpyHostToDevice, s));
        } else {
            std::vector<float> hs(ns * d);
            for (size_t i = 0; i < ns; ++i) std::memcpy(&hs[i * d], x + sample[i] * d, d * sizeof(float));
            HY_CUDA(cudaMemcpyAsync(xs, hs.data(), ns * d * sizeof(float), cudaMemcpyHostToDevice, s));
            HY_CUDA(cudaStreamSynchronize(s));
        }
    }
    return kmeans_device(h, xs, ns, init, lite ? 2 : 20, s);
}

// Build the arena from n device rows x that are already grouped: `order` (an
// array of n row indices, device) lists rows list by list; labels[i] is row
// i's list.  sizes = rows per list.
int build_arena(hy_index* h, const float* x, size_t n, const int32_t* order, const int64_t* labels,
                const std::vector<int32_t>& sizes, cudaStream_t s) {
    const size_t nlist = h->nlist;
    // An index restricted to lists [list_lo, list_hi) stores only their rows
    // (the other lists stay empty); `start` follows the sorted order of all rows.
    const size_t lo = std::min(h->list_lo, nlist), hi = std::min(h->list_hi, nlist);
    const bool ranged = lo > 0 || hi < nlist;
    std::vector<int32_t> kept = sizes;
    if (ranged)
        for (size_t l = 0; l < nlist; ++l)
            if (l < lo || l >= hi) kept[l] = 0;
    h->h_list_size = kept;
    h->h_list_off.assign(nlist + 1, 0);
    std::vector<int64_t> start(nlist + 1, 0);
    size_t held = 0;
    for (size_t l = 0; l < nlist; ++l) {
        start[l + 1] = start[l] + sizes[l];
        held += kept[l];
        // Lists start on 128-row boundaries: a 128-row tensor-core tile (and
        // four 32-row scan tiles) never straddles two lists.
        h->h_list_off[l + 1] = h->h_list_off[l] + (kept[l] + hy::BATCH_ROW_ALIGN - 1) / hy::BATCH_ROW_ALIGN *
                                                      hy::BATCH_ROW_ALIGN;
    }
    h->arena_rows = (size_t)h->h_list_off[nlist];
    const size_t rows_alloc = std::max<size_t>(h->arena_rows, hy::BATCH_ROW_ALIGN);
    h->abf_valid = false;
    h->a8_valid = false;
    h->c2c_valid = false;
    HY_RET(h->codes.ensure(rows_alloc * h->L.row_pitch * sizeof(float)));
    HY_RET(h->ids.ensure(rows_alloc * sizeof(int64_t)));
    HY_RET(h->norms.ensure(rows_alloc * sizeof(float)));
    HY_RET(h->list_off.ensure((nlist + 1) * sizeof(int64_t)));
    HY_RET(h->list_size.ensure(nlist * sizeof(int32_t)));
    HY_RET(h->w_start.ensure((nlist + 1) * sizeof(int64_t)));
    HY_CUDA(cudaMemsetAsync(h->codes.p, 0, rows_alloc * h->L.row_pitch * sizeof(float), s));
    HY_CUDA(cudaMemsetAsync(h->norms.p, 0, rows_alloc * sizeof(float), s));
    HY_CUDA(hy::launch_fill_i64(h->ids.as<int64_t>(), (int64_t)rows_alloc, -1, s));
    HY_CUDA(cudaMemcpyAsync(h->list_off.p, h->h_list_off.data(), (nlist + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemcpyAsync(h->list_size.p, kept.data(), nlist * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemcpyAsync(h->w_start.p, start.data(), (nlist + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    if (n > 0)
        HY_CUDA(hy::launch_scatter(h->L, x, (int64_t)n, order, labels, h->w_start.as<int64_t>(),
                                   h->list_off.as<int64_t>(), ranged ? h->list_size.as<int32_t>() : nullptr,
                                   h->codes.as<float>(), h->ids.as<int64_t>(), h->norms.as<float>(), s));
    HY_CUDA(cudaStreamSynchronize(s));
    h->ntotal = held;
    return HY_OK;
}

int add_impl(hy_index* h, size_t n, const float* x, bool x_on_device, cudaStream_t s) {
    HY_CHECK(h->trained, HY_ERR_STATE, "add: index is not trained (no centroids)");
    HY_CHECK(n < (size_t(1) << 31), HY_ERR_ARG, "add: at most 2^31-1 rows per call");
    const size_t d = h->d, nlist = h->nlist;
    if (n == 0) {
        // The reference returns without touching the lists (src/Index.cpp:583-590).
        return HY_OK;
    }
    const float* xd = x;
    if (!x_on_device) {
        HY_RET(h->w_x.ensure(n * d * sizeof(float)));
        HY_CUDA(cudaMemcpyAsync(h->w_x.p, x, n * d * sizeof(float), cudaMemcpyHostToDevice, s));
        xd = h->w_x.as<float>();
    }
    HY_RET(h->w_lab.ensure(n * sizeof(int64_t)));
    HY_RET(h->w_dist.ensure(n * sizeof(float)));
    HY_RET(assign_rows(h, xd, n, h->w_lab.as<int64_t>(), h->w_dist.as<float>(), s));
    // list sizes
    HY_RET(h->w_cnt.ensure(nlist * sizeof(int32_t)));
    HY_CUDA(cudaMemsetAsync(h->w_cnt.p, 0, nlist * sizeof(int32_t), s));
    HY_CUDA(hy::launch_histogram(h->w_lab.as<int64_t>(), (int64_t)n, h->w_cnt.as<int32_t>(), s));
    std::vector<int32_t> sizes(nlist);
    HY_CUDA(cudaMemcpyAsync(sizes.data(), h->w_cnt.p, nlist * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    // order rows by (list, score to centroid), stable in row id
    HY_RET(h->w_keys.ensure(n * sizeof(uint64_t)));
    HY_RET(h->w_keys2.ensure(n * sizeof(uint64_t)));
    HY_RET(h->w_vals.ensure(n * sizeof(int32_t)));
    HY_RET(h->w_vals2.ensure(n * sizeof(int32_t)));
    HY_CUDA(hy::launch_make_sort_keys(h->w_lab.as<int64_t>(), h->w_dist.as<float>(), (int64_t)n,
                                      h->w_keys.as<uint64_t>(), h->w_vals.as<int32_t>(), s));
    int lbits = 1;
    while ((size_t(1) << lbits) < nlist) ++lbits;
    size_t tmp = 0;
    HY_CUDA(hy::radix_sort_pairs(nullptr, &tmp, h->w_keys.as<uint64_t>(), h->w_keys2.as<uint64_t>(),
                                 h->w_vals.as<int32_t>(), h->w_vals2.as<int32_t>(), (int64_t)n, 32 + lbits, s));
    HY_RET(h->w_sort.ensure(tmp));
    tmp = h->w_sort.bytes;
    HY_CUDA(hy::radix_sort_pairs(h->w_sort.p, &tmp, h->w_keys.as<uint64_t>(), h->w_keys2.as<uint64_t>(),
                                 h->w_vals.as<int32_t>(), h->w_vals2.as<int32_t>(), (int64_t)n, 32 + lbits, s));
    HY_CUDA(cudaStreamSynchronize(s));
    return build_arena(h, xd, n, h->w_vals2.as<int32_t>(), h->w_lab.as<int64_t>(), sizes, s);
}

int check_search_args(hy_index* h, size_t n, size_t k) {
    HY_CHECK(k >= 1 && k <= HY_MAX_K, HY_ERR_ARG, "search: k must be in [1, " + std::to_string(HY_MAX_K) + "]");
    HY_CHECK(h->trained, HY_ERR_STATE, "search: index is not trained (no centroids)");
    HY_CHECK(n < (size_t(1) << 31) / 1, HY_ERR_ARG, "search: too many queries");
    return HY_OK;
}

// Search n device queries with device probe lists (nprobe per query) into
// device D/I.  Runs on stream s; does not synchronise.
// nq_dev (optional): a device count of the queries to search (the first
// *nq_dev of the n); the scan's CTAs then loop over them, one wave of
// query slots per SM.
int scan_and_merge(hy_index* h, size_t n, const float* dq, size_t k, size_t nprobe, const int64_t* dprobes,
                   const uint32_t* init_thr, float* dD, int64_t* dI, cudaStream_t s, bool timed,
                   int64_t* drows = nullptr, const int32_t* nq_dev = nullptr) {
    const int kp = k <= 32 ? 32 : k <= 64 ? 64 : k <= 128 ? 128 : 256;
    int nsplit = 1;
    const size_t target_ctas = 2 * 148;
    if (n < target_ctas) nsplit = (int)std::min<size_t>((target_ctas + n - 1) / n, std::max<size_t>(nprobe, 1));
    while ((nprobe + nsplit - 1) / nsplit > 2048) ++nsplit;
    HY_RET(h->w_parts.ensure(n * nsplit * kp * sizeof(uint64_t)));
    uint32_t* gthr = nullptr;
    if (nsplit > 1) {
        HY_RET(h->w_gthr.ensure(n * sizeof(uint32_t)));
        gthr = h->w_gthr.as<uint32_t>();
        if (init_thr)
            HY_CUDA(cudaMemcpyAsync(gthr, init_thr, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        else
            HY_CUDA(cudaMemsetAsync(gthr, 0xff, n * sizeof(uint32_t), s));
    }
    hy::ScanParams p;
    p.L = h->L;
    p.codes = h->codes.as<float>();
    p.list_off = h->list_off.as<int64_t>();
    p.list_size = h->list_size.as<int32_t>();
    p.q = dq;
    p.probes = dprobes;
    p.init_thr = init_thr;
    p.g_thr = gthr;
    p.out = h->w_parts.as<uint64_t>();
    p.counters = h->w_counters.as<unsigned long long>();
    p.err = h->w_err.as<int>();
    p.nq = (int)n;
    p.nprobe = (int)nprobe;
    p.nsplit = nsplit;
    p.k = (int)k;
    p.metric = h->metric;
    p.prune = 1;
    p.nq_dev = nq_dev;
    if (nq_dev) {
        if (h->nsm == 0) HY_CUDA(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
        p.qgrid = h->nsm;
    }
    if (timed) HY_CUDA(ev_record(h->ev[2], s));
    h->launches += 2 + (nsplit > 1 ? 1 : 0);
    int smem = 0;
    cudaError_t e = hy::launch_scan_plain(p, &smem, s);
    if (e != cudaSuccess)
        return fail(HY_ERR_CUDA, std::string("scan launch (") + std::to_string(smem) + " B shared): " + cudaGetErrorString(e));
    if (timed) HY_CUDA(ev_record(h->ev[3], s));
    HY_CUDA(hy::launch_merge(h->w_parts.as<uint64_t>(), (int)n, nsplit, kp, (int)k, h->metric, h->ids.as<int64_t>(),
                             dD, dI, s, drows, nq_dev));
    if (timed) HY_CUDA(ev_record(h->ev[4], s));
    return HY_OK;
}

// Rows per work item of the list-major scan (32 tiles: four per warp).
constexpr int LM_ROW_SLICE = 1024;

// Whether a plain search of m queries (per chunk) at nprobe runs the
// list-major scan.
bool use_list_major(const hy_index* h, size_t m, size_t nprobe) {
    if (h->plain_scan == HY_PLAIN_QUERY_MAJOR || h->arena_rows == 0 || !hy::list_scan_fits(h->L)) return false;
    if (h->plain_scan == HY_PLAIN_LIST_MAJOR) return true;
    return m * nprobe >= 4 * h->nlist;
}

// The list-major plain scan of m device queries whose probe lists (m x
// nprobe, -1 = skip) and ordered-key thresholds (thr: warm-up values or
// 0xffffffff; lowered in place) are on the device, into D / I: first pass
// over each query's nearest list, the k best keys kept and the threshold
// lowered to the k-th, second pass over the other probed lists, final
// top-k; queries whose candidates overflowed are searched again by the
// query-major scan.  Runs on stream s.
int scan_lists(hy_index* h, size_t m, const float* qq, size_t k, size_t nprobe, const int64_t* probes, uint32_t* thr,
               float* dD, int64_t* dI, cudaStream_t s, bool timed) {
    if (h->nsm == 0) HY_CUDA(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
    const size_t nlist = h->nlist;
    const size_t capq = h->capq;
    const int rs = LM_ROW_SLICE;
    HY_RET(h->b_pcnt.ensure(nlist * sizeof(int32_t)));
    HY_RET(h->b_pfill.ensure(nlist * sizeof(int32_t)));
    HY_RET(h->b_poff.ensure((nlist + 1) * sizeof(int64_t)));
    HY_RET(h->b_pairs.ensure(m * nprobe * sizeof(int32_t)));
    HY_RET(h->b_icnt.ensure(nlist * sizeof(int32_t)));
    HY_RET(h->b_ioff.ensure((nlist + 1) * sizeof(int64_t)));
    HY_RET(h->b_work.ensure(sizeof(unsigned int)));
    HY_RET(h->b_done.ensure_zeroed(sizeof(unsigned int)));
    HY_RET(h->b_cand.ensure(m * capq * sizeof(uint64_t)));
    HY_RET(h->b_ccnt.ensure(m * sizeof(int32_t)));
    HY_RET(h->b_ovf.ensure((m + 1) * sizeof(int32_t)));
    size_t max_slices = 1;
    for (size_t l = 0; l < nlist; ++l)
        max_slices = std::max(max_slices, ((size_t)h->h_list_size[l] + rs - 1) / rs);
    const size_t item_cap = std::min<size_t>((m * nprobe / hy::LM_GROUP + nlist) * max_slices, size_t(4) << 20);
    HY_RET(h->b_items.ensure(item_cap * sizeof(int4)));
    HY_RET(h->b_fq.ensure(m * h->d * sizeof(float)));
    HY_RET(h->b_fpr.ensure(m * nprobe * sizeof(int64_t)));
    HY_RET(h->b_fD.ensure(m * k * sizeof(float)));
    HY_RET(h->b_fI.ensure(m * k * sizeof(int64_t)));
    HY_RET(h->b_fcnt.ensure(sizeof(int32_t)));
    HY_RET(h->b_fbtot.ensure(sizeof(unsigned long long)));
    hy::BatchWork w{};
    w.items = h->b_items.as<int4>();
    w.item_cap = (int64_t)item_cap;
    w.pair_cnt = h->b_pcnt.as<int32_t>();
    w.pair_fill = h->b_pfill.as<int32_t>();
    w.pair_off = h->b_poff.as<int64_t>();
    w.pairs = h->b_pairs.as<int32_t>();
    w.item_cnt = h->b_icnt.as<int32_t>();
    w.item_off = h->b_ioff.as<int64_t>();
    w.work = h->b_work.as<unsigned int>();
    w.done = h->b_done.as<unsigned int>();
    int32_t* ovf = h->b_ovf.as<int32_t>();
    HY_CUDA(cudaMemsetAsync(h->b_ccnt.p, 0, m * sizeof(int32_t), s));
    HY_CUDA(cudaMemsetAsync(ovf, 0, sizeof(int32_t), s));
    hy::ListScanParams p;
    p.L = h->L;
    p.codes = h->codes.as<float>();
    p.list_off = h->list_off.as<int64_t>();
    p.list_size = h->list_size.as<int32_t>();
    p.q = qq;
    p.item_off = w.item_off;
    p.items = w.items;
    p.item_cap = w.item_cap;
    p.pair_off = w.pair_off;
    p.pairs = w.pairs;
    p.pair_cnt = w.pair_cnt;
    p.thr = thr;
    p.cand = h->b_cand.as<uint64_t>();
    p.cand_cnt = h->b_ccnt.as<int32_t>();
    p.work = w.work;
    p.counters = h->w_counters.as<unsigned long long>();
    p.err = h->w_err.as<int>();
    p.nlist = (int)nlist;
    p.rs = rs;
    p.capq = (int)capq;
    p.metric = h->metric;
    p.prune = 1;
    if (h->opt_level & 1) {
        // OPT_TRIANGLE: centroid windows of each (query, list).  Inner
        // product: the reference's cos-bound window.  L2 (the reference's L2
        // triangle is commented out, so its search is unpruned): rows whose
        // distance to the centroid differs from the query's by more than the
        // square root of its threshold cannot reach it, an exact prune that
        // pays when lists are tight balls around their centroids.
        if (!h->c2c_valid) {
            const size_t rows = std::max<size_t>(h->arena_rows, hy::BATCH_ROW_ALIGN);
            HY_RET(h->c2c.ensure(rows * sizeof(float)));
            HY_RET(h->c2c_tile.ensure(rows / 32 * sizeof(float2)));
            HY_CUDA(hy::launch_row_centroid(h->L, h->codes.as<float>(), h->list_off.as<int64_t>(),
                                            h->list_size.as<int32_t>(), (int)nlist, (int64_t)h->arena_rows,
                                            h->cent.as<float>(), h->metric, h->c2c.as<float>(),
                                            h->c2c_tile.as<float2>(), s));
            h->c2c_valid = true;
        }
        p.triangle = 1;
        p.c2c = h->c2c.as<float>();
        p.c2c_tile = h->c2c_tile.as<float2>();
        p.cent = h->cent.as<float>();
    }
    if (timed) HY_CUDA(ev_record(h->ev[2], s));
    // Pass 1: each query's nearest list.
    HY_CUDA(hy::launch_invert_probes(probes, (int)m, (int)nprobe, 0, 1, (int)nlist, h->list_size.as<int32_t>(), rs,
                                     hy::LM_GROUP, w, s));
    HY_CUDA(cudaMemsetAsync(w.work, 0, sizeof(unsigned int), s));
    if (timed) HY_CUDA(ev_record(h->ev[6], s));
    HY_CUDA(hy::launch_list_scan(p, h->nsm, s));
    if (timed) HY_CUDA(ev_record(h->ev[7], s));
    if (timed) h->kev = 1;
    HY_CUDA(hy::launch_list_topk(p.cand, p.cand_cnt, (int)m, (int)capq, (int)k, h->metric, 0, thr, nullptr, nullptr,
                                 nullptr, nullptr, s));
    h->launches += 8;
    if (nprobe > 1) {
        // Pass 2: the other probed lists under the lowered thresholds.
        HY_CUDA(hy::launch_invert_probes(probes, (int)m, (int)nprobe, 1, (int)nprobe, (int)nlist,
                                         h->list_size.as<int32_t>(), rs, hy::LM_GROUP, w, s));
        HY_CUDA(cudaMemsetAsync(w.work, 0, sizeof(unsigned int), s));
        if (timed) HY_CUDA(ev_record(h->ev[8], s));
        HY_CUDA(hy::launch_list_scan(p, h->nsm, s));
        if (timed) HY_CUDA(ev_record(h->ev[9], s));
        if (timed) h->kev = 2;
        h->launches += 7;
    }
    if (timed) HY_CUDA(ev_record(h->ev[3], s));
    HY_CUDA(hy::launch_list_topk(p.cand, p.cand_cnt, (int)m, (int)capq, (int)k, h->metric, 1, thr,
                                 h->ids.as<int64_t>(), dD, dI, ovf, s));
    // Overflowed queries: the query-major scan over the same probe lists.
    HY_CUDA(hy::launch_fb_gather(ovf, qq, probes, (int)nprobe, (int)h->d, (int)m, h->b_fq.as<float>(),
                                 h->b_fpr.as<int64_t>(), h->b_fcnt.as<int32_t>(), s));
    HY_RET(scan_and_merge(h, m, h->b_fq.as<float>(), k, nprobe, h->b_fpr.as<int64_t>(), nullptr, h->b_fD.as<float>(),
                          h->b_fI.as<int64_t>(), s, false, nullptr, h->b_fcnt.as<int32_t>()));
    HY_CUDA(hy::launch_fb_scatter(ovf, h->b_fD.as<float>(), h->b_fI.as<int64_t>(), (int)k, (int)m, dD, dI,
                                  h->b_fbtot.as<unsigned long long>(), s));
    if (timed) HY_CUDA(ev_record(h->ev[4], s));
    h->launches += 3;
    return HY_OK;
}

int ensure_common(hy_index* h) {
    HY_RET(h->w_counters.ensure(4 * sizeof(unsigned long long)));
    HY_RET(h->w_err.ensure(sizeof(int)));
    return HY_OK;
}

int search_bf16_impl(hy_index* h, size_t n, const float* dq, size_t k, float* dD, int64_t* dI, cudaStream_t s,
                     bool timed);

bool learned_on(const hy_index* h) { return h->learned && h->model_ready; }
bool batched_form(const hy_index* h) { return h->form == HY_FORM_BF16 || h->form == HY_FORM_FP8; }

// Chunk of queries whose probes (m x nprobe, best first) and their coarse
// scores (h->m_pscore) are on the device: the probe network predicts each
// query's nprobe and the probes beyond it become -1.
int apply_learned_probes(hy_index* h, size_t m, size_t nprobe, cudaStream_t s, int64_t* probes = nullptr,
                         size_t q0 = 0) {
    if (!probes) probes = h->w_probes.as<int64_t>();
    HY_RET(h->m_total.ensure(sizeof(unsigned long long)));
    // Rows at or past learned_rows keep the fixed nprobe (judged rows).
    const size_t mc = h->learned_rows > q0 ? std::min(m, h->learned_rows - q0) : 0;
    if (mc == 0) return HY_OK;
    HY_CUDA(hy::mlp_infer(h->m_pscore.as<float>(), (int)mc, (int)nprobe, h->m_mu.as<float>(), h->m_sd.as<float>(),
                          h->m_wimg.as<unsigned char>(), h->m_params.as<float>(), h->margin, probes,
                          h->m_total.as<unsigned long long>(), nullptr, h->w_err.as<int>(), s));
    h->launches += 1;
    return HY_OK;
}

// Full device search: coarse quantisation, optional warm-up thresholds, scan,
// merge, in query chunks.
int search_device_impl(hy_index* h, size_t n, const float* dq, size_t k, float* dD, int64_t* dI, cudaStream_t s,
                       bool timed) {
    HY_RET(ensure_common(h));
    HY_CUDA(cudaMemsetAsync(h->w_counters.p, 0, 4 * sizeof(unsigned long long), s));
    h->lm_last = false;
    h->stats.list_major = 0;
    if (batched_form(h) && h->arena_rows > 0) return search_bf16_impl(h, n, dq, k, dD, dI, s, timed);
    const size_t nprobe = std::min(h->nprobe, h->nlist);
    HY_CHECK(nprobe >= 1, HY_ERR_ARG, "search: nprobe must be >= 1");
    HY_CHECK(h->nlist <= 40000, HY_ERR_ARG, "search: nlist above 40000 is not supported by the coarse selector");
    HY_RET(ensure_common(h));
    size_t qc = query_chunk(h->nlist, n);
    // List-major scan: chunks sized so the candidate buffers stay within 2 GiB.
    const bool lm = use_list_major(h, qc, nprobe);
    if (lm) qc = std::min(qc, std::max<size_t>(1, (size_t(2) << 30) / (h->capq * 8)));
    h->lm_last = lm;
    h->stats.list_major = lm ? 1 : 0;
    HY_RET(h->w_scores.ensure(qc * h->nlist * sizeof(float)));
    HY_RET(h->w_probes.ensure(qc * nprobe * sizeof(int64_t)));
    if (learned_on(h)) HY_RET(h->m_pscore.ensure(qc * nprobe * sizeof(float)));
    const bool warm = h->warmup_list > 0 && h->metric == HY_METRIC_L2;
    if (warm || lm) HY_RET(h->w_thr.ensure(qc * sizeof(uint32_t)));
    if (lm) {
        HY_RET(h->b_fbtot.ensure(sizeof(unsigned long long)));
        HY_CUDA(cudaMemsetAsync(h->b_fbtot.p, 0, sizeof(unsigned long long), s));
    }
    for (size_t q0 = 0; q0 < n; q0 += qc) {
        const size_t m = std::min(qc, n - q0);
        h->stats.chunk_queries = m;  // the last chunk's count remains
        const float* qq = dq + q0 * h->d;
        if (timed && q0 == 0) HY_CUDA(ev_record(h->ev[0], s));
        // The list-major scan's counters restart at the last query chunk, the
        // one whose scan launches the kernel events time, so that the
        // executed partial sums and kernel_ms describe the same launches.
        if (lm && q0 > 0 && q0 + m >= n)
            HY_CUDA(cudaMemsetAsync(h->w_counters.p, 0, 4 * sizeof(unsigned long long), s));
        HY_CUDA(hy::launch_coarse_scores(qq, (int)m, h->cent.as<float>(), (int)h->nlist, (int)h->d, h->metric,
                                         h->w_scores.as<float>(), s));
        HY_CUDA(hy::launch_select(h->w_scores.as<float>(), (int)m, (int)h->nlist, (int)nprobe,
                                  h->w_probes.as<int64_t>(), learned_on(h) ? h->m_pscore.as<float>() : nullptr, s));
        h->launches += 2;
        if (learned_on(h)) HY_RET(apply_learned_probes(h, m, nprobe, s, nullptr, q0));
        if (h->q_nprobe) {
            HY_CUDA(hy::launch_cut_probes(h->w_probes.as<int64_t>(), (int)m, (int)nprobe, h->q_nprobe + q0, s));
            h->launches += 1;
        }
        const uint32_t* thr = nullptr;
        if (warm) {
            h->launches += 1;
            const size_t wls = h->warmup_list_size ? h->warmup_list_size : k;
            HY_CHECK(std::min(h->warmup_list, nprobe) * wls <= 32768, HY_ERR_ARG,
                     "presearch: warmup_list * warmup_list_size above 32768");
            HY_CUDA(hy::launch_warmup(h->L, h->codes.as<float>(), h->list_off.as<int64_t>(), h->list_size.as<int32_t>(),
                                      qq, (int)m, h->w_probes.as<int64_t>(), (int)nprobe, (int)k, (int)h->warmup_list,
                                      (int)wls, 1, h->w_thr.as<uint32_t>(), nullptr, h->w_err.as<int>(), s));
            thr = h->w_thr.as<uint32_t>();
        }
        if (timed && q0 == 0) HY_CUDA(ev_record(h->ev[1], s));
        if (lm) {
            if (!warm) HY_CUDA(cudaMemsetAsync(h->w_thr.p, 0xff, m * sizeof(uint32_t), s));
            HY_RET(scan_lists(h, m, qq, k, nprobe, h->w_probes.as<int64_t>(), h->w_thr.as<uint32_t>(), dD + q0 * k,
                              dI + q0 * k, s, timed && q0 + qc >= n));
        } else {
            HY_RET(scan_and_merge(h, m, qq, k, nprobe, h->w_probes.as<int64_t>(), thr, dD + q0 * k, dI + q0 * k, s,
                                  timed && q0 + qc >= n));
        }
    }
    return HY_OK;
}

// The bf16 tensor-core image of the arena, built on first use after add/load.
int ensure_bf16_image(hy_index* h, cudaStream_t s) {
    if (h->form == HY_FORM_FP8) {
        if (h->a8_valid) return HY_OK;
        const size_t rows = std::max<size_t>(h->arena_rows, hy::BATCH_ROW_ALIGN);
        const size_t tiles = rows / hy::BATCH_ROW_ALIGN;
        HY_RET(h->a8.ensure(hy::f8_image_bytes((int64_t)rows, (int)h->d)));
        HY_RET(h->x8aux.ensure(rows * sizeof(float2)));
        HY_RET(h->t8aux.ensure(tiles * sizeof(float2)));
        HY_RET(h->lscale.ensure(h->nlist * sizeof(float)));
        HY_RET(h->tscale.ensure(tiles * sizeof(float)));
        HY_RET(h->tmax.ensure(tiles * sizeof(float)));
        HY_CUDA(hy::launch_to_f8_arena(h->L, h->codes.as<float>(), (int64_t)rows, h->list_off.as<int64_t>(),
                                       h->list_size.as<int32_t>(), (int)h->nlist, h->tmax.as<float>(),
                                       h->lscale.as<float>(), h->tscale.as<float>(), h->a8.p, s));
        HY_CUDA(hy::launch_row_aux(h->L, h->codes.as<float>(), (int64_t)rows, h->tscale.as<float>(),
                                   h->x8aux.as<float2>(), h->t8aux.as<float2>(), s));
        HY_RET(h->txn.ensure(tiles * sizeof(float)));
        HY_CUDA(hy::launch_tile_max(h->norms.as<float>(), (int64_t)rows, h->txn.as<float>(), s));
        h->a8_valid = true;
        return HY_OK;
    }
    if (h->abf_valid) return HY_OK;
    const size_t rows = std::max<size_t>(h->arena_rows, hy::BATCH_ROW_ALIGN);
    HY_RET(h->abf.ensure(hy::bf16_image_bytes((int64_t)rows, (int)h->d)));
    HY_RET(h->xaux.ensure(rows * sizeof(float2)));
    HY_RET(h->taux.ensure(rows / hy::BATCH_ROW_ALIGN * sizeof(float2)));
    HY_CUDA(hy::launch_to_bf16_arena(h->L, h->codes.as<float>(), (int64_t)rows, h->abf.p, s));
    HY_CUDA(hy::launch_row_aux(h->L, h->codes.as<float>(), (int64_t)rows, nullptr, h->xaux.as<float2>(), h->taux.as<float2>(),
                               s));
    HY_RET(h->txn.ensure(rows / hy::BATCH_ROW_ALIGN * sizeof(float)));
    HY_CUDA(hy::launch_tile_max(h->norms.as<float>(), (int64_t)rows, h->txn.as<float>(), s));
    // Exactness certificate of the image (see launch_prep_queries).
    HY_RET(h->b_cert.ensure(2 * sizeof(int32_t)));
    const int32_t init[2] = {1, 0};
    HY_CUDA(cudaMemcpyAsync(h->b_cert.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    HY_CUDA(hy::launch_arena_integral(h->codes.as<float>(), (int64_t)(rows * h->L.row_pitch), h->norms.as<float>(),
                                      (int64_t)rows, h->b_cert.as<int>(), reinterpret_cast<unsigned int*>(h->b_cert.as<int>() + 1),
                                      s));
    int32_t cert[2] = {0, 0};
    HY_CUDA(cudaMemcpyAsync(cert, h->b_cert.p, sizeof(cert), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaStreamSynchronize(s));
    float mx;
    std::memcpy(&mx, &cert[1], sizeof(float));
    h->arena_maxxn = cert[0] ? mx : -1.0f;
    h->abf_valid = true;
    return HY_OK;
}

// Whether the bf16 form's coarse step runs on the tensor cores (the
// conditions launch_coarse_refine's shared memory and select width need).
bool coarse_on_tensor(const hy_index* h, size_t nprobe) {
    return h->coarse_mode == HY_COARSE_TENSOR && h->form == HY_FORM_BF16 && nprobe <= 256 && h->d <= 256 &&
           hy::batched_group_size((int)h->d, false) > 0;
}

int ensure_centroid_image(hy_index* h, cudaStream_t s) {
    if (h->cimg_valid) return HY_OK;
    const size_t rows = (h->nlist + hy::BATCH_ROW_ALIGN - 1) / hy::BATCH_ROW_ALIGN * hy::BATCH_ROW_ALIGN;
    HY_RET(h->c_img.ensure(hy::bf16_split_image_bytes((int64_t)rows, (int)h->d)));
    HY_RET(h->c_aux.ensure(rows * sizeof(float2)));
    HY_RET(h->c_taux.ensure(rows / hy::BATCH_ROW_ALIGN * sizeof(float2)));
    HY_RET(h->c_norm.ensure(rows * sizeof(float)));
    HY_RET(h->c_off.ensure(2 * sizeof(int64_t)));
    HY_RET(h->c_size.ensure(sizeof(int32_t)));
    HY_CUDA(hy::launch_centroid_image(h->cent.as<float>(), (int)h->nlist, (int)h->d, h->c_img.p, h->c_aux.as<float2>(),
                                      h->c_taux.as<float2>(), h->c_norm.as<float>(), s));
    h->cimg_valid = true;
    return HY_OK;
}

// Coarse step on the tensor cores for m queries whose bf16 image and
// {|q|^2, |q|, |q~|, |q - q~|} are in b_qb / b_qn: one dense batched launch
// over the centroid index, then the exact m best per query.
int coarse_tensor(hy_index* h, size_t m, const float* qq, size_t nprobe, int64_t* probes, float* pscore,
                  cudaStream_t s) {
    HY_RET(ensure_centroid_image(h, s));
    const int nlist = (int)h->nlist;
    const int qg = hy::batched_group_size((int)h->d, false);
    const int ngroups = (int)((m + qg - 1) / qg);
    // Row slices of a launch over the first `rows` centroids: enough to give
    // every SM an item, each at most 2048 rows.
    auto slicing = [&](int rows, int* rs_out) {
        const int tiles = (rows + 127) / 128;
        int ns = std::min(tiles, std::max(1, (h->nsm + ngroups - 1) / ngroups));
        ns = std::max(ns, (tiles + 15) / 16);
        const int rs = (tiles + ns - 1) / ns * 128;
        *rs_out = rs;
        return (rows + rs - 1) / rs;
    };
    int rs_full;
    const int ns_full = slicing(nlist, &rs_full);
    HY_RET(h->c_pcnt.ensure(sizeof(int32_t)));
    HY_RET(h->c_poff.ensure(2 * sizeof(int64_t)));
    HY_RET(h->c_pairs.ensure(m * sizeof(int32_t)));
    HY_RET(h->c_ioff.ensure(2 * sizeof(int64_t)));
    HY_RET(h->c_items.ensure((size_t)ngroups * ns_full * sizeof(int4)));
    HY_RET(h->c_work.ensure(sizeof(unsigned int)));
    HY_RET(h->c_cand.ensure(m * nlist * sizeof(float2)));
    HY_RET(h->c_ccnt.ensure(m * sizeof(int32_t)));
    hy::BatchWork w{};
    w.items = h->c_items.as<int4>();
    w.pair_cnt = h->c_pcnt.as<int32_t>();
    w.pair_off = h->c_poff.as<int64_t>();
    w.pairs = h->c_pairs.as<int32_t>();
    w.item_off = h->c_ioff.as<int64_t>();
    w.work = h->c_work.as<unsigned int>();
    w.cand = h->c_cand.as<uint64_t>();
    w.cand_cnt = h->c_ccnt.as<int32_t>();
    hy::BatchedLaunch b;
    b.abf = h->c_img.p;
    b.list_off = h->c_off.as<int64_t>();
    b.list_size = h->c_size.as<int32_t>();
    b.xn = h->c_norm.as<float>();
    b.tile_aux = h->c_taux.as<float2>();
    b.xaux = h->c_aux.as<float2>();
    b.qb = h->b_qb.p;
    b.qaux = h->b_qn.as<float4>();
    b.thr = h->b_thr.as<float>();
    b.nlist = 1;
    b.d = (int)h->d;
    b.metric = h->metric;
    b.nsm = h->nsm;
    b.qg = qg;
    b.f8 = false;
    b.ksplit = true;
    if (nlist <= 2048) {
        // Every (query, centroid) score, then the exact best.
        w.item_cap = (int64_t)ngroups * ns_full;
        HY_CUDA(hy::launch_coarse_items((int)m, nlist, ngroups, ns_full, h->c_off.as<int64_t>(),
                                        h->c_size.as<int32_t>(), w, s));
        b.rs = rs_full;
        b.capq = nlist;
        b.dense_max = nlist;
        HY_CUDA(hy::launch_batched_scan(b, w, h->w_err.as<int>(), s));
        HY_CUDA(hy::launch_coarse_refine(reinterpret_cast<float2*>(h->c_cand.p), (int)m, nlist, qq,
                                         h->cent.as<float>(), h->c_norm.as<float>(), h->c_aux.as<float2>(),
                                         h->b_qn.as<float4>(), (int)h->d, h->metric, (int)nprobe, probes, pscore,
                                         h->w_err.as<int>(), s));
        h->launches += 3;
        return HY_OK;
    }
    // More lists: a dense launch over the first S centroids bounds each
    // query's nprobe-th best score (b_thr); a thresholded launch over all
    // centroids emits the keys that can reach it (stride nlist, no
    // overflow); the keys are selected and re-scored exactly.
    const int S = 1024;
    int rs_a;
    const int ns_a = slicing(S, &rs_a);
    w.item_cap = (int64_t)ngroups * ns_a;
    HY_CUDA(hy::launch_coarse_items((int)m, S, ngroups, ns_a, h->c_off.as<int64_t>(), h->c_size.as<int32_t>(), w, s));
    b.rs = rs_a;
    b.capq = S;
    b.dense_max = S;
    HY_CUDA(hy::launch_batched_scan(b, w, h->w_err.as<int>(), s));
    HY_CUDA(hy::launch_coarse_thr(reinterpret_cast<const float2*>(h->c_cand.p), (int)m, S, (int)nprobe,
                                  h->c_norm.as<float>(), h->c_aux.as<float2>(), h->b_qn.as<float4>(), (int)h->d,
                                  h->metric, h->b_thr.as<float>(), s));
    w.item_cap = (int64_t)ngroups * ns_full;
    HY_CUDA(hy::launch_coarse_items((int)m, nlist, ngroups, ns_full, h->c_off.as<int64_t>(), h->c_size.as<int32_t>(),
                                    w, s));
    HY_CUDA(cudaMemsetAsync(w.cand_cnt, 0, m * sizeof(int32_t), s));
    b.rs = rs_full;
    b.capq = nlist;
    b.dense_max = 0;
    HY_CUDA(hy::launch_batched_scan(b, w, h->w_err.as<int>(), s));
    HY_CUDA(hy::launch_coarse_refine_keys(h->c_cand.as<uint64_t>(), w.cand_cnt, (int)m, nlist, qq, h->cent.as<float>(),
                                          h->c_norm.as<float>(), h->c_aux.as<float2>(), h->b_qn.as<float4>(),
                                          (int)h->d, h->metric, (int)nprobe, probes, pscore, h->w_err.as<int>(), s));
    h->launches += 6;
    return HY_OK;
}

// Batched bf16 search of n device queries: coarse quantisation, warm-up
// thresholds, probe inversion, the persistent tensor-core scan and the exact
// re-rank, in query chunks sized so the candidate buffers stay within 2 GiB.
int search_bf16_impl(hy_index* h, size_t n, const float* dq, size_t k, float* dD, int64_t* dI, cudaStream_t s,
                     bool timed) {
    const size_t nprobe = std::min(h->nprobe, h->nlist);
    HY_CHECK(nprobe >= 1, HY_ERR_ARG, "search: nprobe must be >= 1");
    HY_CHECK(h->nlist <= 40000, HY_ERR_ARG, "search: nlist above 40000 is not supported by the coarse selector");
    HY_RET(ensure_common(h));
    HY_RET(ensure_bf16_image(h, s));
    if (h->nsm == 0) HY_CUDA(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
    const size_t capq = h->capq;
    size_t qc = std::min(query_chunk(h->nlist, n), std::max<size_t>(1, (size_t(2) << 30) / (capq * 8)));
    qc = std::min(qc, n);
    const bool f8 = h->form == HY_FORM_FP8;
    const size_t nkb = f8 ? (h->d + 127) / 128 : (h->d + 63) / 64;  // 128-byte k-blocks per row
    const int qg = hy::batched_group_size((int)h->d, f8);
    HY_CHECK(qg > 0, HY_ERR_ARG, "search: d too large for the tensor-core form");
    const size_t nlist = h->nlist;
    HY_RET(h->w_scores.ensure(qc * nlist * sizeof(float)));
    HY_RET(h->w_probes.ensure(qc * nprobe * sizeof(int64_t)));
    if (learned_on(h)) HY_RET(h->m_pscore.ensure(qc * nprobe * sizeof(float)));
    HY_RET(h->w_thr.ensure(qc * sizeof(uint32_t)));
    HY_RET(h->b_thr.ensure(qc * sizeof(float)));
    HY_RET(h->b_qb.ensure(qc * nkb * 128));
    if (f8) HY_RET(h->b_qs.ensure(qc * sizeof(float)));
    HY_RET(h->b_qn.ensure(qc * sizeof(float4)));
    HY_RET(h->b_qx.ensure(qc * sizeof(int32_t)));
    HY_RET(h->b_pcnt.ensure(nlist * sizeof(int32_t)));
    HY_RET(h->b_pfill.ensure(nlist * sizeof(int32_t)));
    HY_RET(h->b_poff.ensure((nlist + 1) * sizeof(int64_t)));
    HY_RET(h->b_pairs.ensure(qc * nprobe * sizeof(int32_t)));
    HY_RET(h->b_icnt.ensure(nlist * sizeof(int32_t)));
    HY_RET(h->b_ioff.ensure((nlist + 1) * sizeof(int64_t)));
    HY_RET(h->b_work.ensure(sizeof(unsigned int)));
    HY_RET(h->b_done.ensure_zeroed(sizeof(unsigned int)));
    HY_RET(h->b_cand.ensure(qc * capq * sizeof(uint64_t)));
    HY_RET(h->b_ccnt.ensure(qc * sizeof(int32_t)));
    HY_RET(h->b_ovf.ensure((qc + 1) * sizeof(int32_t)));
    HY_RET(h->b_big.ensure(3 * (qc + 1) * sizeof(int32_t)));
    // Exact fallback on the device: every overflowed query of a chunk is
    // searched again by the plain scan over the same probe lists.
    const size_t fbcap = qc;
    HY_RET(h->b_fq.ensure(fbcap * h->d * sizeof(float)));
    HY_RET(h->b_fpr.ensure(fbcap * nprobe * sizeof(int64_t)));
    HY_RET(h->b_fD.ensure(fbcap * k * sizeof(float)));
    HY_RET(h->b_fI.ensure(fbcap * k * sizeof(int64_t)));
    HY_RET(h->b_fcnt.ensure(sizeof(int32_t)));
    HY_RET(h->b_fbtot.ensure(sizeof(unsigned long long)));
    HY_CUDA(cudaMemsetAsync(h->b_fbtot.p, 0, sizeof(unsigned long long), s));
    // Warm-up for the bf16 form: its threshold only bounds the first pass
    // (each query's nearest list), so three lists suffice by default.  A
    // query whose nearest list has between k and dense_max rows needs none:
    // the first pass scans that list densely and the tightening step takes
    // the k-th smallest bound over all of its rows.
    const int dense_max = (int)std::min<size_t>(capq, hy::DENSE_MAX);
    const size_t wl = h->warmup_list ? std::min<size_t>(h->warmup_list, 3) : 3;
    const size_t wls = h->warmup_list_size ? h->warmup_list_size : k;
    HY_CHECK(std::min(wl, nprobe) * wls <= 32768, HY_ERR_ARG, "presearch: warmup_list * warmup_list_size above 32768");
    // Item descriptors: an upper bound on the item count from host-known
    // sizes (groups <= pairs/128 + lists, slices per list <= the largest
    // list's), capped at 4M; items beyond the cap are decoded by search.
    size_t max_slices = 1;
    for (size_t l = 0; l < nlist; ++l)
        max_slices = std::max(max_slices, ((size_t)h->h_list_size[l] + h->row_slice - 1) / h->row_slice);
    // Queries per group of each pass (hy_index_set_group_size): by default
    // the smallest of 64 / 128 holding four times the pass's expected
    // queries per list (measured on 1M x 128 at about 10 queries per list:
    // 64 ahead of 128 and 32).  The first pass has one list per query; the
    // second the rest of the fixed nprobe, or of the probe model's held-out
    // mean.
    auto pass_group = [&](double pairs) {
        if (h->group_size) return std::min(h->group_size, qg);
        const double per_list = pairs / (double)nlist;
        int g = 64;
        while (g < qg && g < 4.0 * per_list) g *= 2;
        return std::min(g, qg);
    };
    const double np_rest =
        (learned_on(h) && h->learned_mean > 0) ? std::max(0.0, h->learned_mean - 1.0) : (double)(nprobe - 1);
    const int qg1 = pass_group((double)qc);
    const int qg2 = pass_group((double)qc * np_rest);
    const size_t item_cap =
        std::min<size_t>((qc / qg1 + qc * nprobe / qg2 + 2 * nlist) * max_slices, size_t(4) << 20);
    HY_RET(h->b_items.ensure(item_cap * sizeof(int4)));
    hy::BatchWork w;
    w.items = h->b_items.as<int4>();
    w.item_cap = (int64_t)item_cap;
    w.pair_cnt = h->b_pcnt.as<int32_t>();
    w.pair_fill = h->b_pfill.as<int32_t>();
    w.pair_off = h->b_poff.as<int64_t>();
    w.pairs = h->b_pairs.as<int32_t>();
    w.item_cnt = h->b_icnt.as<int32_t>();
    w.item_off = h->b_ioff.as<int64_t>();
    w.work = h->b_work.as<unsigned int>();
    w.done = h->b_done.as<unsigned int>();
    w.cand = h->b_cand.as<uint64_t>();
    w.cand_cnt = h->b_ccnt.as<int32_t>();
    w.big = h->b_big.as<int32_t>();
    w.big2 = w.big + (qc + 1);
    w.rest = w.big2 + (qc + 1);
    for (size_t q0 = 0; q0 < n; q0 += qc) {
        const size_t m = std::min(qc, n - q0);
        h->stats.chunk_queries = m;  // the last chunk's count remains
        const float* qq = dq + q0 * h->d;
        w.overflow = h->b_ovf.as<int32_t>();  // [0] = count, then chunk-local query ids
        HY_CUDA(cudaMemsetAsync(w.overflow, 0, sizeof(int32_t), s));
        if (timed && q0 == 0) HY_CUDA(ev_record(h->ev[0], s));
        HY_CUDA(hy::launch_prep_queries(qq, (int)m, (int)h->d, h->b_qb.p, h->b_qn.as<float4>(),
                                        f8 ? h->b_qs.as<float>() : nullptr, s, f8 ? -1.0f : h->arena_maxxn,
                                        f8 ? nullptr : h->b_qx.as<int32_t>()));
        if (coarse_on_tensor(h, nprobe)) {
            HY_RET(coarse_tensor(h, m, qq, nprobe, h->w_probes.as<int64_t>(),
                                 learned_on(h) ? h->m_pscore.as<float>() : nullptr, s));
        } else {
            HY_CUDA(hy::launch_coarse_scores(qq, (int)m, h->cent.as<float>(), (int)nlist, (int)h->d, h->metric,
                                             h->w_scores.as<float>(), s));
            HY_CUDA(hy::launch_select(h->w_scores.as<float>(), (int)m, (int)nlist, (int)nprobe,
                                      h->w_probes.as<int64_t>(), learned_on(h) ? h->m_pscore.as<float>() : nullptr, s));
            h->launches += 2;
        }
        if (learned_on(h)) HY_RET(apply_learned_probes(h, m, nprobe, s, nullptr, q0));
        if (h->q_nprobe) {
            HY_CUDA(hy::launch_cut_probes(h->w_probes.as<int64_t>(), (int)m, (int)nprobe, h->q_nprobe + q0, s));
            h->launches += 1;
        }
        if (h->metric == HY_METRIC_L2) {
            HY_CUDA(hy::launch_warmup(h->L, h->codes.as<float>(), h->list_off.as<int64_t>(), h->list_size.as<int32_t>(),
                                      qq, (int)m, h->w_probes.as<int64_t>(), (int)nprobe, (int)k, (int)wl, (int)wls, 1,
                                      h->w_thr.as<uint32_t>(), h->b_thr.as<float>(), h->w_err.as<int>(), s, (int)k,
                                      dense_max));
        } else {
            // Inner products have no warm-up threshold in the reference: the
            // first pass's dense lists bound the pass after it; the other
            // lists' candidate buffers hold every probed row.
            HY_CUDA(hy::launch_fill_f32(h->b_thr.as<float>(), (int64_t)m, INFINITY, s));
        }
        if (timed && q0 == 0) HY_CUDA(ev_record(h->ev[1], s));
        HY_CUDA(cudaMemsetAsync(w.cand_cnt, 0, m * sizeof(int32_t), s));
        if (timed && q0 + qc >= n) HY_CUDA(ev_record(h->ev[2], s));
        hy::BatchedLaunch b;
        b.abf = f8 ? h->a8.p : h->abf.p;
        b.list_off = h->list_off.as<int64_t>();
        b.list_size = h->list_size.as<int32_t>();
        b.xn = h->norms.as<float>();
        b.tile_aux = f8 ? h->t8aux.as<float2>() : h->taux.as<float2>();
        b.xaux = f8 ? h->x8aux.as<float2>() : h->xaux.as<float2>();
        b.lscale = f8 ? h->lscale.as<float>() : nullptr;
        b.qscale = f8 ? h->b_qs.as<float>() : nullptr;
        b.f8 = f8;
        b.qg = qg1;
        b.qb = h->b_qb.p;
        b.qaux = h->b_qn.as<float4>();
        b.thr = h->b_thr.as<float>();
        b.nlist = (int)nlist;
        b.d = (int)h->d;
        b.rs = (int)h->row_slice;
        b.capq = (int)capq;
        b.metric = h->metric;
        b.nsm = h->nsm;
        // Pass 1: each query's nearest list, densely (every row) when it has
        // at most dense_max rows, else under the warm-up threshold; the
        // threshold is then tightened to the k-th smallest candidate upper
        // bound; pass 2: the remaining probed lists under the tight threshold.
        const bool last = timed && q0 + qc >= n;
        HY_CUDA(hy::launch_invert_probes(h->w_probes.as<int64_t>(), (int)m, (int)nprobe, 0, 1, (int)nlist,
                                         h->list_size.as<int32_t>(), (int)h->row_slice, qg1, w, s));
        if (last) HY_CUDA(ev_record(h->ev[6], s));
        b.dense_max = dense_max;
        HY_CUDA(hy::launch_batched_scan(b, w, h->w_err.as<int>(), s));
        b.dense_max = 0;
        if (last) HY_CUDA(ev_record(h->ev[7], s));
        if (last) h->kev = 1;
        hy::DenseFirst df;
        df.probes = h->w_probes.as<int64_t>();
        df.nprobe = (int)nprobe;
        df.list_size = h->list_size.as<int32_t>();
        df.list_off = h->list_off.as<int64_t>();
        df.dense_max = dense_max;
        df.tile_aux = f8 ? h->t8aux.as<float2>() : h->taux.as<float2>();
        df.tile_xn = h->txn.as<float>();
        HY_CUDA(hy::launch_tighten(h->norms.as<float>(), f8 ? h->x8aux.as<float2>() : h->xaux.as<float2>(),
                                   h->b_qn.as<float4>(), (int)m, w, (int)capq, (int)k, h->metric, (int)h->d, f8,
                                   h->nsm, h->b_thr.as<float>(), s, df));
        if (nprobe > 1) {
            HY_CUDA(hy::launch_invert_probes(h->w_probes.as<int64_t>(), (int)m, (int)nprobe, 1, (int)nprobe,
                                             (int)nlist, h->list_size.as<int32_t>(), (int)h->row_slice, qg2, w, s));
            b.qg = qg2;
            if (last) HY_CUDA(ev_record(h->ev[8], s));
            HY_CUDA(hy::launch_batched_scan(b, w, h->w_err.as<int>(), s));
            if (last) HY_CUDA(ev_record(h->ev[9], s));
            if (last) h->kev = 2;
        }
        if (timed && q0 + qc >= n) HY_CUDA(ev_record(h->ev[3], s));
        const int rmax = f8 ? (int)std::min<size_t>(h->oversample * k, 4096) : 0;
        HY_CUDA(hy::launch_rerank(h->L, h->codes.as<float>(), h->ids.as<int64_t>(), h->norms.as<float>(),
                                  f8 ? h->x8aux.as<float2>() : h->xaux.as<float2>(), h->b_qn.as<float4>(), qq, (int)m,
                                  w, 0, (int)capq, (int)k, rmax, h->metric, f8, h->nsm, dD + q0 * k, dI + q0 * k, s,
                                  f8 ? nullptr : h->b_qx.as<int32_t>()));
        if (timed && q0 + qc >= n) HY_CUDA(ev_record(h->ev[4], s));
        const int fb = (int)std::min<size_t>(m, fbcap);
        HY_CUDA(hy::launch_fb_gather(w.overflow, qq, h->w_probes.as<int64_t>(), (int)nprobe, (int)h->d, fb,
                                     h->b_fq.as<float>(), h->b_fpr.as<int64_t>(), h->b_fcnt.as<int32_t>(), s));
        HY_RET(scan_and_merge(h, (size_t)fb, h->b_fq.as<float>(), k, nprobe, h->b_fpr.as<int64_t>(), nullptr,
                              h->b_fD.as<float>(), h->b_fI.as<int64_t>(), s, false, nullptr, h->b_fcnt.as<int32_t>()));
        HY_CUDA(hy::launch_fb_scatter(w.overflow, h->b_fD.as<float>(), h->b_fI.as<int64_t>(), (int)k, fb, dD + q0 * k,
                                      dI + q0 * k, h->b_fbtot.as<unsigned long long>(), s));
        h->launches += 3;
        h->launches += nprobe > 1 ? 24 : 18;
    }
    return HY_OK;
}

// Device times of the phases and of the scan kernel's launches, from the
// events the last timed search recorded (they must have completed).
void collect_times(hy_index* h) {
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
    h->stats.coarse_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]);
    h->stats.scan_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[3], h->ev[4]);
    h->stats.merge_ms = ms;
    if (h->kev > 0) {
        double km = 0.0;
        for (int i = 0; i < h->kev; ++i) {
            cudaEventElapsedTime(&ms, h->ev[6 + 2 * i], h->ev[7 + 2 * i]);
            km += ms;
        }
        h->stats.kernel_ms = km;
        h->stats.kernel_launches = (uint64_t)h->kev;
    } else {
        h->stats.kernel_ms = h->stats.scan_ms;
        h->stats.kernel_launches = 1;
    }
    h->kev = 0;
    h->times_pending = false;
}

// End of a host-pointer call: the device status (error flag, scan
// counters, learned nprobe total, fallback counters) comes back in one
// pinned block with the stream's single synchronisation.
int finish_host_call(hy_index* h, cudaStream_t s, bool timed, size_t n, size_t nprobe) {
    if (!h->hstat) HY_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&h->hstat), sizeof(HostStatus), cudaHostAllocDefault));
    HostStatus* st = h->hstat;
    *st = HostStatus{};
    HY_CUDA(cudaMemcpyAsync(&st->err, h->w_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaMemcpyAsync(st->counters, h->w_counters.p, sizeof(st->counters), cudaMemcpyDeviceToHost, s));
    if (h->m_total.p)
        HY_CUDA(cudaMemcpyAsync(&st->learned_total, h->m_total.p, sizeof(st->learned_total), cudaMemcpyDeviceToHost, s));
    if (h->b_fbtot.p) HY_CUDA(cudaMemcpyAsync(&st->fallback, h->b_fbtot.p, sizeof(st->fallback), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaStreamSynchronize(s));
    if (st->err != 0) {
        const int err = st->err;
        cudaMemset(h->w_err.p, 0, sizeof(int));
        return fail(err == HY_ERR_TIMEOUT ? HY_ERR_TIMEOUT : HY_ERR_CUDA, "device reported an error in the scan kernel");
    }
    h->stats.nq = n;
    h->stats.pairs = n * nprobe;
    h->stats.tile_blocks = st->counters[0];
    h->stats.tile_blocks_max = st->counters[1];
    h->stats.seg_sums = st->counters[2];
    h->stats.seg_sums_max = st->counters[3];
    h->stats.launches = h->launches;
    h->launches = 0;
    if (timed) collect_times(h);
    h->kev = 0;
    return HY_OK;
}

int reset_counters(hy_index* h, cudaStream_t s) {
    HY_RET(ensure_common(h));
    h->launches = 0;
    HY_RET(h->m_total.ensure(sizeof(unsigned long long)));
    HY_CUDA(cudaMemsetAsync(h->m_total.p, 0, sizeof(unsigned long long), s));
    HY_CUDA(cudaMemsetAsync(h->w_counters.p, 0, 4 * sizeof(unsigned long long), s));
    return HY_OK;
}

void drop_graph(hy_index* h) {
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->gexec = nullptr;
    h->graph = nullptr;
}

// The device-pointer search, through a CUDA graph in graph mode: the first
// call with a new (buffers, sizes, stream, index state) runs normally (every
// buffer reaches its size), then captures the same launch sequence; later
// identical calls replay it with one cudaGraphLaunch.  The legacy default
// stream cannot be captured: such calls run the graph on the handle's stream,
// ordered after and before the default stream's work by events.
int run_device_search(hy_index* h, size_t n, const float* dq, size_t k, float* dD, int64_t* dI, cudaStream_t s) {
    h->stats.graph_replayed = 0;
    h->ev = h->ev_direct;
    if (!h->graph_on) return search_device_impl(h, n, dq, k, dD, dI, s, true);
    const hy_index::GraphKey key{h->epoch, n, k, h->nprobe, dq, dD, dI, h->q_nprobe, s, h->learned_rows, h->learned};
    cudaStream_t run = s ? s : h->stream;
    if (h->gexec && key == h->gkey) {
        if (!s) {
            HY_CUDA(cudaEventRecord(h->gev[0], nullptr));
            HY_CUDA(cudaStreamWaitEvent(h->stream, h->gev[0], 0));
        }
        HY_CUDA(cudaGraphLaunch(h->gexec, run));
        h->ev = h->ev_graph;  // the replay recorded the graph's timing events
        if (!s) {
            HY_CUDA(cudaEventRecord(h->gev[1], h->stream));
            HY_CUDA(cudaStreamWaitEvent(nullptr, h->gev[1], 0));
        }
        h->launches = h->graph_kernels;
        h->kev = h->graph_kev;
        h->stats.graph_replayed = 1;
        return HY_OK;
    }
    HY_RET(search_device_impl(h, n, dq, k, dD, dI, s, true));
    const uint64_t launches = h->launches;
    const int kev = h->kev;
    drop_graph(h);
    HY_CUDA(cudaStreamBeginCapture(run, cudaStreamCaptureModeThreadLocal));
    h->launches = 0;
    h->ev = h->ev_graph;
    const int rc = search_device_impl(h, n, dq, k, dD, dI, run, true);
    h->ev = h->ev_direct;  // this call's times come from the direct run
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(run, &g);
    if (rc != HY_OK || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        h->launches = launches;
        h->kev = kev;
        if (rc != HY_OK) return rc;
        return fail(HY_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&h->gexec, g, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(g);
        h->gexec = nullptr;
        return fail(HY_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    h->graph = g;
    h->gkey = key;
    h->graph_kernels = h->launches;
    h->graph_kev = h->kev;
    h->launches = launches;
    h->kev = kev;
    return HY_OK;
}

// Fallback accounting of a bf16 host-pointer search: every overflowed query
// was answered again on the device by the plain scan.  After
// finish_host_call (its status block holds the fallback counter).
int bf16_fallback(hy_index* h) {
    h->stats.fallback_queries = h->hstat->fallback;
    return HY_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

const char* hy_last_error(void) { return g_err.c_str(); }

const char* hy_version(void) { return "hy 0.1 (sm_100a)"; }

int hy_index_create(size_t d, size_t nlist, size_t nprobe, int metric, int opt_level, size_t dim_blocks, int device,
                    hy_index** out) {
    HY_CHECK(out != nullptr, HY_ERR_ARG, "create: out is NULL");
    *out = nullptr;
    HY_CHECK(d >= 1 && d <= 4096, HY_ERR_ARG, "create: d must be in [1, 4096]");
    HY_CHECK(nlist >= 1 && nlist <= (size_t(1) << 24), HY_ERR_ARG, "create: nlist must be in [1, 2^24]");
    HY_CHECK(metric == HY_METRIC_L2 || metric == HY_METRIC_IP, HY_ERR_ARG, "create: metric must be 0 (IP) or 1 (L2)");
    HY_CHECK(opt_level >= 0 && opt_level <= 7, HY_ERR_ARG, "create: invalid opt_level");
    if (dim_blocks == 0) dim_blocks = 4;
    HY_CHECK(dim_blocks <= HY_MAX_DIM_BLOCKS, HY_ERR_ARG, "create: dim_blocks above HY_MAX_DIM_BLOCKS");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(HY_ERR_CUDA, std::string("create: no CUDA device available (") + cudaGetErrorString(e) + ")");
    HY_CHECK(device >= 0 && device < ndev, HY_ERR_ARG, "create: device ordinal out of range");
    auto* h = new (std::nothrow) hy_index();
    HY_CHECK(h != nullptr, HY_ERR_OOM, "create: out of host memory");
    h->device = device;
    h->d = d;
    h->nlist = nlist;
    h->nprobe = nprobe;
    h->metric = metric;
    h->opt_level = opt_level;
    h->dim_blocks = std::min(dim_blocks, d);
    h->L = make_layout((int)d, (int)h->dim_blocks);
    int rc = set_device(h);
    if (rc == HY_OK) {
        e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        for (int i = 0; e == cudaSuccess && i < 10; ++i) e = cudaEventCreate(&h->ev_direct[i]);
        for (int i = 0; e == cudaSuccess && i < 10; ++i) e = cudaEventCreate(&h->ev_graph[i]);
        if (e != cudaSuccess) rc = fail(HY_ERR_CUDA, std::string("create: ") + cudaGetErrorString(e));
    }
    if (rc == HY_OK) rc = ensure_common(h);
    if (rc == HY_OK) {
        cudaMemset(h->w_err.p, 0, sizeof(int));
    }
    if (rc != HY_OK) {
        hy_index_destroy(h);
        return rc;
    }
    *out = h;
    return HY_OK;
}

int hy_index_destroy(hy_index* h) {
    if (!h) return HY_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    DevBuf* bufs[] = {&h->cent,   &h->list_off, &h->list_size, &h->ids,    &h->codes,   &h->norms,  &h->w_q,
                      &h->w_scores, &h->w_probes, &h->w_thr,   &h->w_gthr, &h->w_parts, &h->w_D,    &h->w_I,
                      &h->w_f,    &h->w_counters, &h->w_err,   &h->w_x,    &h->w_lab,   &h->w_dist, &h->w_keys,
                      &h->w_keys2, &h->w_vals,  &h->w_vals2,   &h->w_sort, &h->w_start, &h->w_sums, &h->w_cnt,
                      &h->w_rows, &h->w_xn};
    for (DevBuf* b : bufs) b->release();
    drop_graph(h);
    for (auto& ev : h->ev_direct)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : h->ev_graph)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : h->gev)
        if (ev) cudaEventDestroy(ev);
    if (h->hstat) cudaFreeHost(h->hstat);
    if (h->hjudge) cudaFreeHost(h->hjudge);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return HY_OK;
}

int hy_index_info(const hy_index* h, hy_index_info_t* out) {
    HY_CHECK(h && out, HY_ERR_ARG, "info: NULL argument");
    out->d = h->d;
    out->nlist = h->nlist;
    out->nprobe = h->nprobe;
    out->metric = h->metric;
    out->opt_level = h->opt_level;
    out->dim_blocks = h->dim_blocks;
    out->ntotal = h->ntotal;
    out->arena_rows = h->arena_rows;
    out->trained = h->trained ? 1 : 0;
    out->device = h->device;
    out->form = h->form;
    out->learned = learned_on(h) ? 1 : 0;
    out->capq = h->capq;
    out->row_slice = h->row_slice;
    return HY_OK;
}

int hy_index_train(hy_index* h, size_t n, const float* x, int lite) {
    HY_CHECK(h && (x || n == 0), HY_ERR_ARG, "train: NULL argument");
    h->epoch++;  // a captured search graph no longer matches
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(set_device(h));
    return train_impl(h, n, x, false, lite, h->stream);
}

int hy_index_train_device(hy_index* h, size_t n, const float* dx, int lite, void* stream) {
    HY_CHECK(h && (dx || n == 0), HY_ERR_ARG, "train: NULL argument");
    h->epoch++;  // a captured search graph no longer matches
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(set_device(h));
    return train_impl(h, n, dx, true, lite, static_cast<cudaStream_t>(stream));
}

int hy_index_set_centroids(hy_index* h, const float* c) {
    HY_CHECK(h && c, HY_ERR_ARG, "set_centroids: NULL argument");
    h->epoch++;  // a captured search graph no longer matches
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(set_device(h));
    const size_t bytes = h->nlist * h->d * sizeof(float);
    HY_RET(h->cent.ensure(bytes));
    h->h_cent.assign(c, c + h->nlist * h->d);
    HY_CUDA(cudaMemcpy(h->cent.p, c, bytes, cudaMemcpyHostToDevice));
    h->trained = true;
    h->cimg_valid = false;
    h->c2c_valid = false;
    return HY_OK;
}

int hy_index_get_centroids(const hy_index* h, float* c) {
    HY_CHECK(h && c, HY_ERR_ARG, "get_centroids: NULL argument");
    HY_CHECK(h->trained, HY_ERR_STATE, "get_centroids: index is not trained");
    std::memcpy(c, h->h_cent.data(), h->nlist * h->d * sizeof(float));
    return HY_OK;
}

int hy_index_add(hy_index* h, size_t n, const float* x) {
    HY_CHECK(h && (x || n == 0), HY_ERR_ARG, "add: NULL argument");
    h->epoch++;  // a captured search graph no longer matches
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(set_device(h));
    return add_impl(h, n, x, false, h->stream);
}

int hy_index_add_device(hy_index* h, size_t n, const float* dx, void* stream) {
    HY_CHECK(h && (dx || n == 0), HY_ERR_ARG, "add: NULL argument");
    h->epoch++;  // a captured search graph no longer matches
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(set_device(h));
    return add_impl(h, n, dx, true, static_cast<cudaStream_t>(stream));
}

int hy_index_set_opt_level(hy_index* h, int opt_level) {
    HY_CHECK(h, HY_ERR_ARG, "set_opt_level: NULL handle");
    HY_CHECK(opt_level >= 0 && opt_level <= 7, HY_ERR_ARG, "set_opt_level: invalid opt_level");
    std::lock_guard<std::mutex> g(h->mu);
    h->epoch++;  // a captured search graph no longer matches
    h->opt_level = opt_level;
    return HY_OK;
}

int hy_index_set_nprobe(hy_index* h, size_t nprobe) {
    HY_CHECK(h, HY_ERR_ARG, "set_nprobe: NULL handle");
    h->epoch++;  // a captured search graph no longer matches
    HY_CHECK(nprobe >= 1, HY_ERR_ARG, "set_nprobe: nprobe must be >= 1");
    h->nprobe = nprobe;
    return HY_OK;
}

int hy_index_set_form(hy_index* h, int form) {
    HY_CHECK(h, HY_ERR_ARG, "set_form: NULL handle");
    h->epoch++;  // a captured search graph no longer matches
    HY_CHECK(form == HY_FORM_PLAIN || form == HY_FORM_BF16 || form == HY_FORM_FP8, HY_ERR_ARG,
             "set_form: unknown form");
    HY_CHECK(form == HY_FORM_PLAIN || hy::batched_group_size((int)h->d, form == HY_FORM_FP8) > 0, HY_ERR_ARG,
             "set_form: d too large for the tensor-core forms (bf16: d <= 768, e4m3: d <= 1536)");
    h->form = form;
    return HY_OK;
}

int hy_index_set_plain_scan(hy_index* h, int mode) {
    HY_CHECK(h, HY_ERR_ARG, "set_plain_scan: NULL handle");
    HY_CHECK(mode == HY_PLAIN_AUTO || mode == HY_PLAIN_QUERY_MAJOR || mode == HY_PLAIN_LIST_MAJOR, HY_ERR_ARG,
             "set_plain_scan: unknown mode");
    std::lock_guard<std::mutex> g(h->mu);
    h->epoch++;  // a captured search graph no longer matches
    h->plain_scan = mode;
    return HY_OK;
}

int hy_index_set_group_size(hy_index* h, int qg) {
    HY_CHECK(h, HY_ERR_ARG, "set_group_size: NULL handle");
    HY_CHECK(qg == 0 || qg == 32 || qg == 64 || qg == 128, HY_ERR_ARG, "set_group_size: qg must be 0, 32, 64 or 128");
    h->epoch++;  // a captured search graph no longer matches
    h->group_size = qg;
    return HY_OK;
}

int hy_index_set_batch_params(hy_index* h, size_t capq, size_t oversample, size_t row_slice) {
    HY_CHECK(h, HY_ERR_ARG, "set_batch_params: NULL handle");
    h->epoch++;  // a captured search graph no longer matches
    if (capq) {
        HY_CHECK(capq >= 64 && capq <= 12288, HY_ERR_ARG, "set_batch_params: capq must be in [64, 12288]");
        h->capq = capq;
    }
    if (oversample) h->oversample = oversample;
    if (row_slice) {
        HY_CHECK(row_slice % hy::BATCH_ROW_ALIGN == 0 && row_slice <= 2048, HY_ERR_ARG,
                 "set_batch_params: row_slice must be a multiple of 128, at most 2048");
        h->row_slice = row_slice;
    }
    return HY_OK;
}

int hy_index_set_coarse(hy_index* h, int mode) {
    HY_CHECK(h, HY_ERR_ARG, "set_coarse: NULL handle");
    HY_CHECK(mode == HY_COARSE_EXACT || mode == HY_COARSE_TENSOR, HY_ERR_ARG, "set_coarse: unknown mode");
    h->epoch++;  // a captured search graph no longer matches
    h->coarse_mode = mode;
    return HY_OK;
}

int hy_index_presearch(hy_index* h, size_t warmup_list, size_t warmup_list_size) {
    HY_CHECK(h, HY_ERR_ARG, "presearch: NULL handle");
    h->epoch++;  // a captured search graph no longer matches
    h->warmup_list = warmup_list;
    h->warmup_list_size = warmup_list_size;
    return HY_OK;
}

int hy_index_search_device(hy_index* h, size_t n, const float* dq, size_t k, float* dD, int64_t* dI, void* stream) {
    HY_CHECK(h && (n == 0 || (dq && dD && dI)), HY_ERR_ARG, "search: NULL argument");
    std::lock_guard<std::mutex> g(h->mu);
    if (n == 0) return HY_OK;
    HY_RET(check_search_args(h, n, k));
    HY_RET(set_device(h));
    // The caller's stream as given: NULL is the CUDA default stream.
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HY_RET(ensure_common(h));
    h->launches = 0;
    HY_RET(run_device_search(h, n, dq, k, dD, dI, s));
    h->stats.launches = h->launches;
    h->stats.nq = n;
    h->times_pending = true;
    return HY_OK;
}

int hy_index_autotune(hy_index* h, size_t n, const float* q, size_t k, int reps, float* report) {
    HY_CHECK(h && q && n >= 1 && reps >= 1, HY_ERR_ARG, "autotune: need a handle, queries and reps >= 1");
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(check_search_args(h, n, k));
    HY_CHECK(batched_form(h), HY_ERR_STATE, "autotune: select the bf16 or e4m3 form first");
    HY_RET(set_device(h));
    h->ev = h->ev_direct;
    h->epoch++;
    cudaStream_t s = h->stream;
    HY_RET(ensure_common(h));
    HY_RET(h->w_q.ensure(n * h->d * sizeof(float)));
    HY_RET(h->w_D.ensure(n * k * sizeof(float)));
    HY_RET(h->w_I.ensure(n * k * sizeof(int64_t)));
    HY_CUDA(cudaMemcpy(h->w_q.p, q, n * h->d * sizeof(float), cudaMemcpyHostToDevice));
    // Candidate work shapes: rows per work item (the list-side tile extent
    // of an item) x candidate slots per query.  Every shape returns the same
    // exact answer; the fastest is kept.
    const size_t slices[3] = {512, 1024, 2048};
    const size_t capqs[2] = {8192, 12288};  // the first pass scans lists of up to capq rows densely
    const size_t keep_rs = h->row_slice, keep_capq = h->capq;
    std::vector<int64_t> ref_I;
    std::vector<int64_t> got_I(n * k);
    double best = 1e30;
    size_t best_rs = keep_rs, best_capq = keep_capq;
    int c = 0;
    for (size_t rs : slices)
        for (size_t cq : capqs) {
            h->row_slice = rs;
            h->capq = cq;
            int rc = search_device_impl(h, n, h->w_q.as<float>(), k, h->w_D.as<float>(), h->w_I.as<int64_t>(), s, false);
            if (rc == HY_OK) {
                HY_CUDA(ev_record(h->ev[6], s));
                for (int r = 0; r < reps && rc == HY_OK; ++r)
                    rc = search_device_impl(h, n, h->w_q.as<float>(), k, h->w_D.as<float>(), h->w_I.as<int64_t>(), s,
                                            false);
                HY_CUDA(ev_record(h->ev[7], s));
            }
            if (rc != HY_OK) {
                h->row_slice = keep_rs;
                h->capq = keep_capq;
                return rc;
            }
            HY_CUDA(cudaStreamSynchronize(s));
            float ms = 0.0f;
            HY_CUDA(cudaEventElapsedTime(&ms, h->ev[6], h->ev[7]));
            ms /= (float)reps;
            HY_CUDA(cudaMemcpy(got_I.data(), h->w_I.p, n * k * sizeof(int64_t), cudaMemcpyDeviceToHost));
            if (ref_I.empty()) ref_I = got_I;
            const bool same = got_I == ref_I;
            if (report) {
                report[3 * c] = (float)rs;
                report[3 * c + 1] = (float)cq;
                report[3 * c + 2] = same ? ms : -ms;
            }
            if (same && ms < best) {
                best = ms;
                best_rs = rs;
                best_capq = cq;
            }
            ++c;
        }
    h->row_slice = best_rs;
    h->capq = best_capq;
    h->launches = 0;
    h->kev = 0;
    return HY_OK;
}

int hy_index_set_list_range(hy_index* h, size_t lo, size_t hi) {
    HY_CHECK(h, HY_ERR_ARG, "set_list_range: NULL handle");
    h->epoch++;  // a captured search graph no longer matches
    HY_CHECK(lo < hi && hi <= h->nlist, HY_ERR_ARG, "set_list_range: need 0 <= lo < hi <= nlist");
    h->list_lo = lo;
    h->list_hi = hi;
    return HY_OK;
}

int hy_merge_topk(const float* dD, const int64_t* dI, size_t parts, size_t n, size_t k, int metric, float* dDout,
                  int64_t* dIout, void* stream) {
    HY_CHECK(n == 0 || (dD && dI && dDout && dIout), HY_ERR_ARG, "merge_topk: NULL argument");
    HY_CHECK(parts >= 1 && parts <= 64 && k >= 1 && k <= HY_MAX_K && parts * k <= 8192, HY_ERR_ARG,
             "merge_topk: need 1 <= parts <= 64, 1 <= k <= 256 and parts * k <= 8192");
    HY_CHECK(metric == HY_METRIC_L2 || metric == HY_METRIC_IP, HY_ERR_ARG, "merge_topk: unknown metric");
    if (n == 0) return HY_OK;
    HY_CHECK(n < (size_t(1) << 31), HY_ERR_ARG, "merge_topk: too many queries");
    HY_CUDA(hy::launch_merge_parts(dD, dI, (int)parts, (int)n, (int)k, metric, dDout, dIout,
                                   static_cast<cudaStream_t>(stream)));
    return HY_OK;
}

int hy_index_set_graph(hy_index* h, int enabled) {
    HY_CHECK(h, HY_ERR_ARG, "set_graph: NULL handle");
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(set_device(h));
    if (enabled && !h->gev[0]) {
        HY_CUDA(cudaEventCreateWithFlags(&h->gev[0], cudaEventDisableTiming));
        HY_CUDA(cudaEventCreateWithFlags(&h->gev[1], cudaEventDisableTiming));
    }
    if (!enabled) drop_graph(h);
    h->graph_on = enabled != 0;
    return HY_OK;
}

}  // extern "C"

namespace {

// The host-pointer search of one batch: upload, device search, download,
// bf16 overflow fallback, statistics.
int search_host(hy_index* h, size_t n, const float* q, size_t k, float* D, int64_t* I,
                const std::vector<int64_t>* judge_rows = nullptr, int64_t* jI = nullptr) {
    cudaStream_t s = h->stream;
    h->ev = h->ev_direct;
    // Judged rows (learned form) ride along at the end of the batch: the
    // same queries again, with the fixed nprobe (the learned cut stops at
    // row n).
    const size_t m = judge_rows ? judge_rows->size() : 0;
    const size_t nt = n + m;
    HY_RET(h->w_q.ensure(nt * h->d * sizeof(float)));
    HY_RET(h->w_D.ensure(nt * k * sizeof(float)));
    HY_RET(h->w_I.ensure(nt * k * sizeof(int64_t)));
    HY_RET(reset_counters(h, s));
    const size_t d = h->d;
    HY_CUDA(cudaMemcpyAsync(h->w_q.p, q, n * d * sizeof(float), cudaMemcpyHostToDevice, s));
    if (m) {
        HY_RET(h->w_jrows.ensure(m * sizeof(int64_t)));
        HY_CUDA(cudaMemcpyAsync(h->w_jrows.p, judge_rows->data(), m * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        HY_CUDA(hy::launch_gather_rows(h->w_q.as<float>(), h->w_jrows.as<int64_t>(), (int64_t)m, (int)d,
                                       h->w_q.as<float>() + n * d, s));
    }
    h->learned_rows = n;
    // Graph mode replays the captured search (the workspace pointers and
    // the stream are the handle's own, so repeated calls of one shape match).
    const int rc = h->graph_on
                       ? run_device_search(h, nt, h->w_q.as<float>(), k, h->w_D.as<float>(), h->w_I.as<int64_t>(), s)
                       : search_device_impl(h, nt, h->w_q.as<float>(), k, h->w_D.as<float>(), h->w_I.as<int64_t>(), s,
                                            true);
    h->learned_rows = SIZE_MAX;
    HY_RET(rc);
    // The results go back before the status checks (one synchronisation for
    // both); a batch searched again below is copied again.
    HY_CUDA(cudaMemcpyAsync(D, h->w_D.p, n * k * sizeof(float), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaMemcpyAsync(I, h->w_I.p, n * k * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    if (m) HY_CUDA(cudaMemcpyAsync(jI, h->w_I.as<int64_t>() + n * k, m * k * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    HY_RET(finish_host_call(h, s, true, nt, std::min(h->nprobe, h->nlist)));
    h->stats.nq = n;
    h->stats.fallback_queries = 0;
    h->stats.mean_nprobe = (double)std::min(h->nprobe, h->nlist);
    if (learned_on(h)) h->stats.mean_nprobe = (double)h->hstat->learned_total / (double)n;
    if ((batched_form(h) || h->lm_last) && h->arena_rows > 0) HY_RET(bf16_fallback(h));
    return HY_OK;
}

// The learned nprobe is judged on every batch: every (1/judge_fraction)-th
// query is searched a second time with the fixed nprobe in the same device
// pass, and the learned results' recall@10 against those is measured; below
// the target, the whole batch is searched again with the fixed nprobe.
int search_learned_judged(hy_index* h, size_t n, const float* q, size_t k, float* D, int64_t* I) {
    const size_t step = std::max<size_t>(1, (size_t)std::lround(1.0 / std::max(1e-6f, h->judge_fraction)));
    std::vector<int64_t> rows;
    for (size_t i = 0; i < n; i += step) rows.push_back((int64_t)i);
    const size_t m = rows.size();
    // The judged rows' results land in pinned memory (a pageable target
    // would make their copy a separate staged transfer).
    if (h->hjudge_cap < m * k) {
        if (h->hjudge) cudaFreeHost(h->hjudge);
        h->hjudge = nullptr;
        h->hjudge_cap = 0;
        HY_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&h->hjudge), m * k * sizeof(int64_t), cudaHostAllocDefault));
        h->hjudge_cap = m * k;
    }
    const int64_t* sI = h->hjudge;
    HY_RET(search_host(h, n, q, k, D, I, &rows, h->hjudge));
    const size_t kk = std::min<size_t>(10, k);
    size_t hit = 0, tot = 0;
    for (size_t i = 0; i < m; ++i) {
        const int64_t* a = I + rows[i] * k;
        const int64_t* b = &sI[i * k];
        for (size_t j = 0; j < kk; ++j) {
            if (b[j] < 0) continue;
            ++tot;
            for (size_t t = 0; t < kk; ++t)
                if (a[t] == b[j]) {
                    ++hit;
                    break;
                }
        }
    }
    const double recall = tot ? (double)hit / (double)tot : 1.0;
    h->stats.judge_recall = recall;
    h->stats.learned_fallback = 0;
    if (recall < h->judge_recall) {
        h->learned = 0;
        const int rc2 = search_host(h, n, q, k, D, I);
        h->learned = 1;
        HY_RET(rc2);
        h->stats.judge_recall = recall;
        h->stats.learned_fallback = 1;
    }
    return HY_OK;
}

// Chunked exact labelling for the probe network: for every query, coarse
// scores of its P best lists (features) and its stop label.
int probe_training_data(hy_index* h, size_t n, const float* q, size_t P, size_t kl, float* X, float* lab, float* S,
                        cudaStream_t s) {
    const size_t qc = std::min<size_t>(query_chunk(h->nlist, n), 8192);
    HY_RET(ensure_common(h));
    HY_RET(h->w_q.ensure(qc * h->d * sizeof(float)));
    HY_RET(h->w_scores.ensure(qc * h->nlist * sizeof(float)));
    HY_RET(h->w_probes.ensure(qc * P * sizeof(int64_t)));
    HY_RET(h->m_pscore.ensure(qc * P * sizeof(float)));
    HY_RET(h->t_D.ensure(qc * kl * sizeof(float)));
    HY_RET(h->t_I.ensure(qc * kl * sizeof(int64_t)));
    HY_RET(h->t_rows.ensure(qc * kl * sizeof(int64_t)));
    HY_RET(h->t_t.ensure(qc * sizeof(float)));
    HY_RET(h->m_X.ensure(qc * hy::MLP_IN * sizeof(float)));
    for (size_t q0 = 0; q0 < n; q0 += qc) {
        const size_t m = std::min(qc, n - q0);
        HY_CUDA(cudaMemcpyAsync(h->w_q.p, q + q0 * h->d, m * h->d * sizeof(float), cudaMemcpyHostToDevice, s));
        HY_CUDA(hy::launch_coarse_scores(h->w_q.as<float>(), (int)m, h->cent.as<float>(), (int)h->nlist, (int)h->d,
                                         h->metric, h->w_scores.as<float>(), s));
        HY_CUDA(hy::launch_select(h->w_scores.as<float>(), (int)m, (int)h->nlist, (int)P, h->w_probes.as<int64_t>(),
                                  h->m_pscore.as<float>(), s));
        HY_CUDA(hy::launch_probe_features(h->m_pscore.as<float>(), (int)m, (int)P, nullptr, nullptr,
                                          h->m_X.as<float>(), s));
        HY_RET(scan_and_merge(h, m, h->w_q.as<float>(), kl, P, h->w_probes.as<int64_t>(), nullptr, h->t_D.as<float>(),
                              h->t_I.as<int64_t>(), s, false, h->t_rows.as<int64_t>()));
        HY_CUDA(hy::launch_stop_labels(h->t_rows.as<int64_t>(), (int)m, (int)kl, h->w_probes.as<int64_t>(), (int)P,
                                       h->list_off.as<int64_t>(), (int)h->nlist, h->t_t.as<float>(), s));
        HY_CUDA(cudaMemcpyAsync(X + q0 * hy::MLP_IN, h->m_X.p, m * hy::MLP_IN * sizeof(float), cudaMemcpyDeviceToHost, s));
        HY_CUDA(cudaMemcpyAsync(lab + q0, h->t_t.p, m * sizeof(float), cudaMemcpyDeviceToHost, s));
        HY_CUDA(cudaMemcpyAsync(S + q0 * P, h->m_pscore.p, m * P * sizeof(float), cudaMemcpyDeviceToHost, s));
        HY_CUDA(cudaStreamSynchronize(s));
    }
    return HY_OK;
}

}  // namespace

extern "C" {

int hy_index_search(hy_index* h, size_t n, const float* q, size_t k, float* D, int64_t* I) {
    HY_CHECK(h && (n == 0 || (q && D && I)), HY_ERR_ARG, "search: NULL argument");
    std::lock_guard<std::mutex> g(h->mu);
    if (n == 0) return HY_OK;
    HY_RET(check_search_args(h, n, k));
    HY_RET(set_device(h));
    if (learned_on(h) && h->judge_fraction > 0) return search_learned_judged(h, n, q, k, D, I);
    HY_RET(search_host(h, n, q, k, D, I));
    h->stats.judge_recall = -1.0;
    h->stats.learned_fallback = 0;
    return HY_OK;
}

int hy_index_search_nprobes(hy_index* h, size_t n, const float* q, size_t k, const int32_t* nprobes, float* D,
                            int64_t* I) {
    HY_CHECK(h && (n == 0 || (q && nprobes && D && I)), HY_ERR_ARG, "search_nprobes: NULL argument");
    std::lock_guard<std::mutex> g(h->mu);
    if (n == 0) return HY_OK;
    HY_RET(check_search_args(h, n, k));
    int32_t mx = 0;
    double sum = 0.0;
    for (size_t i = 0; i < n; ++i) {
        HY_CHECK(nprobes[i] >= 1, HY_ERR_ARG, "search_nprobes: every nprobe must be >= 1");
        const int32_t c = (int32_t)std::min<size_t>((size_t)nprobes[i], h->nlist);
        mx = std::max(mx, c);
        sum += c;
    }
    HY_RET(set_device(h));
    HY_RET(h->w_np.ensure(n * sizeof(int32_t)));
    HY_CUDA(cudaMemcpy(h->w_np.p, nprobes, n * sizeof(int32_t), cudaMemcpyHostToDevice));
    const size_t keep = h->nprobe;
    h->nprobe = (size_t)mx;
    h->q_nprobe = h->w_np.as<int32_t>();
    const int rc = search_host(h, n, q, k, D, I);
    h->q_nprobe = nullptr;
    h->nprobe = keep;
    HY_RET(rc);
    if (!learned_on(h)) h->stats.mean_nprobe = sum / (double)n;
    h->stats.judge_recall = -1.0;
    h->stats.learned_fallback = 0;
    return HY_OK;
}

int hy_index_search_nprobes_device(hy_index* h, size_t n, const float* dq, size_t k, const int32_t* dnprobes,
                                   size_t max_nprobe, float* dD, int64_t* dI, void* stream) {
    HY_CHECK(h && (n == 0 || (dq && dnprobes && dD && dI)), HY_ERR_ARG, "search_nprobes: NULL argument");
    HY_CHECK(max_nprobe >= 1, HY_ERR_ARG, "search_nprobes: max_nprobe must be >= 1");
    std::lock_guard<std::mutex> g(h->mu);
    if (n == 0) return HY_OK;
    HY_RET(check_search_args(h, n, k));
    HY_RET(set_device(h));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HY_RET(ensure_common(h));
    h->launches = 0;
    const size_t keep = h->nprobe;
    h->nprobe = std::min(max_nprobe, h->nlist);
    h->q_nprobe = dnprobes;
    const int rc = run_device_search(h, n, dq, k, dD, dI, s);
    h->q_nprobe = nullptr;
    h->nprobe = keep;
    HY_RET(rc);
    h->stats.launches = h->launches;
    h->stats.nq = n;
    h->times_pending = true;
    return HY_OK;
}

int hy_index_train_probe_model(hy_index* h, size_t n, const float* q, size_t max_nprobe, size_t k_label, int epochs,
                               float lr, float coverage, float* report) {
    HY_CHECK(h && q && n >= 100, HY_ERR_ARG, "train_probe_model: need a handle and at least 100 queries");
    h->epoch++;  // a captured search graph no longer matches
    HY_CHECK(k_label >= 1 && k_label <= HY_MAX_K && epochs >= 1 && lr > 0 && coverage > 0 && coverage < 1, HY_ERR_ARG,
             "train_probe_model: bad k_label / epochs / lr / coverage");
    std::lock_guard<std::mutex> g(h->mu);
    HY_CHECK(h->trained && !h->h_list_size.empty(), HY_ERR_STATE, "train_probe_model: build the index first");
    HY_RET(set_device(h));
    cudaStream_t s = h->stream;
    const size_t P = std::max<size_t>(1, std::min(max_nprobe, h->nlist));
    // 1. features and exact stop labels
    std::vector<float> X(n * hy::MLP_IN), lab(n), S(n * P);
    HY_RET(probe_training_data(h, n, q, P, k_label, X.data(), lab.data(), S.data(), s));
    const size_t ntr = std::max<size_t>(1, n * 9 / 10), nva = n - ntr;
    std::vector<float> t(n);
    for (size_t i = 0; i < n; ++i) t[i] = std::log2(std::max(1.0f, lab[i]));
    // 2. feature standardisation from the training part
    std::vector<float> mu(hy::MLP_IN, 0.0f), sd(hy::MLP_IN, 0.0f);
    for (size_t i = 0; i < ntr; ++i)
        for (int f = 0; f < hy::MLP_IN; ++f) mu[f] += X[i * hy::MLP_IN + f];
    for (int f = 0; f < hy::MLP_IN; ++f) mu[f] /= (float)ntr;
    for (size_t i = 0; i < ntr; ++i)
        for (int f = 0; f < hy::MLP_IN; ++f) {
            const float dlt = X[i * hy::MLP_IN + f] - mu[f];
            sd[f] += dlt * dlt;
        }
    for (int f = 0; f < hy::MLP_IN; ++f) sd[f] = std::sqrt(sd[f] / (float)ntr) + 1e-6f;
    for (size_t i = 0; i < n; ++i)
        for (int f = 0; f < hy::MLP_IN; ++f) X[i * hy::MLP_IN + f] = (X[i * hy::MLP_IN + f] - mu[f]) / sd[f];
    // 3. initial weights (uniform, scaled by fan-in + fan-out; fixed seed)
    std::vector<float> params(hy::MLP_NPARAM, 0.0f);
    std::mt19937 rng(1234);
    auto fill = [&](int off, int fin, int fout) {
        const float a = std::sqrt(6.0f / (float)(fin + fout));
        std::uniform_real_distribution<float> U(-a, a);
        for (int i = 0; i < fin * fout; ++i) params[off + i] = U(rng);
    };
    fill(hy::MLP_W1, hy::MLP_IN, hy::MLP_H);
    fill(hy::MLP_W2, hy::MLP_H, hy::MLP_H);
    fill(hy::MLP_W3, hy::MLP_H, 1);
    const int B = 256;
    HY_RET(h->m_params.ensure(hy::MLP_NPARAM * sizeof(float)));
    HY_RET(h->t_grads.ensure(hy::MLP_NPARAM * sizeof(float)));
    HY_RET(h->t_am.ensure(hy::MLP_NPARAM * sizeof(float)));
    HY_RET(h->t_av.ensure(hy::MLP_NPARAM * sizeof(float)));
    HY_RET(h->t_X.ensure(n * hy::MLP_IN * sizeof(float)));
    HY_RET(h->t_t.ensure(n * sizeof(float)));
    HY_RET(h->t_Xb.ensure((size_t)B * hy::MLP_IN * sizeof(float)));
    HY_RET(h->t_tb.ensure((size_t)B * sizeof(float)));
    HY_RET(h->t_dy.ensure((size_t)B * sizeof(float)));
    HY_RET(h->m_y.ensure(std::max<size_t>(B, 8192) * sizeof(float)));
    HY_RET(h->t_loss.ensure(sizeof(float)));
    HY_RET(h->t_perm.ensure(ntr * sizeof(int64_t)));
    HY_RET(h->m_work.ensure(hy::mlp_work_floats(8192) * sizeof(float)));
    HY_CUDA(cudaMemcpyAsync(h->m_params.p, params.data(), params.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemsetAsync(h->t_am.p, 0, hy::MLP_NPARAM * sizeof(float), s));
    HY_CUDA(cudaMemsetAsync(h->t_av.p, 0, hy::MLP_NPARAM * sizeof(float), s));
    HY_CUDA(cudaMemcpyAsync(h->t_X.p, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemcpyAsync(h->t_t.p, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    hy::MlpWork w;
    hy::mlp_work_bind(w, h->m_work.as<float>(), B);
    // 4. Adam on mini-batches of 256, reshuffled every epoch
    std::vector<int64_t> perm(ntr);
    std::iota(perm.begin(), perm.end(), 0);
    int step = 0;
    double last_loss = 0.0;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        HY_CUDA(cudaMemcpyAsync(h->t_perm.p, perm.data(), ntr * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        HY_CUDA(cudaStreamSynchronize(s));
        double eloss = 0.0;
        int nb = 0;
        for (size_t b0 = 0; b0 + B <= ntr; b0 += B) {
            const int64_t* idx = h->t_perm.as<int64_t>() + b0;
            HY_CUDA(hy::launch_gather_rows(h->t_X.as<float>(), idx, B, hy::MLP_IN, h->t_Xb.as<float>(), s));
            HY_CUDA(hy::launch_gather_rows(h->t_t.as<float>(), idx, B, 1, h->t_tb.as<float>(), s));
            HY_CUDA(hy::mlp_forward(h->m_params.as<float>(), B, h->t_Xb.as<float>(), w, h->m_y.as<float>(), s));
            HY_CUDA(hy::mlp_mse(B, h->m_y.as<float>(), h->t_tb.as<float>(), h->t_dy.as<float>(), h->t_loss.as<float>(), s));
            HY_CUDA(hy::mlp_backward(h->m_params.as<float>(), B, h->t_Xb.as<float>(), w, h->t_dy.as<float>(),
                                     h->t_grads.as<float>(), s));
            HY_CUDA(hy::mlp_adam(h->m_params.as<float>(), h->t_grads.as<float>(), h->t_am.as<float>(), h->t_av.as<float>(),
                                 ++step, lr, s));
            if (ep == epochs - 1) {
                float lv = 0.0f;
                HY_CUDA(cudaMemcpyAsync(&lv, h->t_loss.p, sizeof(float), cudaMemcpyDeviceToHost, s));
                HY_CUDA(cudaStreamSynchronize(s));
                eloss += lv;
                ++nb;
            }
        }
        if (ep == epochs - 1) last_loss = nb ? eloss / nb : 0.0;
    }
    // 5. margin: the `coverage` quantile of (label - prediction) on held-out
    // queries, so that fraction of them gets at least its stop point.
    const size_t nv = nva ? nva : ntr;
    const size_t v0 = nva ? ntr : 0;
    // Held-out predictions come from the inference kernel the search uses.
    std::vector<float> yv(nv);
    HY_RET(h->m_mu.ensure(hy::MLP_IN * sizeof(float)));
    HY_RET(h->m_sd.ensure(hy::MLP_IN * sizeof(float)));
    HY_CUDA(cudaMemcpy(h->m_mu.p, mu.data(), hy::MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    HY_CUDA(cudaMemcpy(h->m_sd.p, sd.data(), hy::MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    HY_RET(h->m_wimg.ensure(hy::mlp_wimg_bytes()));
    HY_CUDA(hy::mlp_pack(h->m_params.as<float>(), h->m_wimg.as<unsigned char>(), s));
    HY_RET(h->m_pscore.ensure(nv * P * sizeof(float)));
    HY_RET(h->m_y.ensure(nv * sizeof(float)));
    HY_CUDA(cudaMemcpyAsync(h->m_pscore.p, S.data() + v0 * P, nv * P * sizeof(float), cudaMemcpyHostToDevice, s));
    HY_CUDA(hy::mlp_infer(h->m_pscore.as<float>(), (int)nv, (int)P, h->m_mu.as<float>(), h->m_sd.as<float>(),
                          h->m_wimg.as<unsigned char>(), h->m_params.as<float>(), 0.0f, nullptr, nullptr,
                          h->m_y.as<float>(), h->w_err.as<int>(), s));
    HY_CUDA(cudaMemcpyAsync(yv.data(), h->m_y.p, nv * sizeof(float), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaStreamSynchronize(s));
    std::vector<float> resid(nv);
    for (size_t i = 0; i < nv; ++i) resid[i] = t[v0 + i] - yv[i];
    std::vector<float> sorted = resid;
    std::sort(sorted.begin(), sorted.end());
    const float margin = sorted[std::min(nv - 1, (size_t)std::ceil(coverage * (double)nv) - 1)];
    double mean_np = 0.0, covered = 0.0, mean_lab = 0.0;
    for (size_t i = 0; i < nv; ++i) {
        const float e = std::exp2(std::min(yv[i] + margin, 30.0f));
        const double np = std::max(1.0, std::min((double)P, std::ceil((double)e)));
        mean_np += np;
        covered += np >= lab[v0 + i] ? 1.0 : 0.0;
        mean_lab += lab[v0 + i];
    }
    h->margin = margin;
    h->model_P = (int)P;
    h->model_ready = true;
    h->learned_mean = mean_np / (double)nv;
    if (report) {
        report[0] = (float)last_loss;
        report[1] = (float)(covered / (double)nv);
        report[2] = (float)(mean_np / (double)nv);
        report[3] = (float)(mean_lab / (double)nv);
    }
    return HY_OK;
}

int hy_index_set_learned(hy_index* h, int enabled, float judge_fraction, float judge_recall) {
    HY_CHECK(h, HY_ERR_ARG, "set_learned: NULL handle");
    h->epoch++;  // a captured search graph no longer matches
    HY_CHECK(!enabled || h->model_ready, HY_ERR_STATE, "set_learned: no probe model (train or set one first)");
    HY_CHECK(judge_fraction >= 0 && judge_fraction <= 1 && judge_recall >= 0 && judge_recall <= 1, HY_ERR_ARG,
             "set_learned: judge_fraction and judge_recall must be in [0, 1]");
    h->learned = enabled ? 1 : 0;
    h->judge_fraction = judge_fraction;
    h->judge_recall = judge_recall;
    return HY_OK;
}

size_t hy_probe_model_size(void) { return (size_t)hy::MLP_NPARAM + 2 * hy::MLP_IN + 2; }

int hy_index_get_probe_model(const hy_index* hc, float* out) {
    HY_CHECK(hc && out, HY_ERR_ARG, "get_probe_model: NULL argument");
    HY_CHECK(hc->model_ready, HY_ERR_STATE, "get_probe_model: no probe model");
    hy_index* h = const_cast<hy_index*>(hc);
    HY_RET(set_device(h));
    HY_CUDA(cudaMemcpy(out, h->m_params.p, hy::MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    HY_CUDA(cudaMemcpy(out + hy::MLP_NPARAM, h->m_mu.p, hy::MLP_IN * sizeof(float), cudaMemcpyDeviceToHost));
    HY_CUDA(cudaMemcpy(out + hy::MLP_NPARAM + hy::MLP_IN, h->m_sd.p, hy::MLP_IN * sizeof(float), cudaMemcpyDeviceToHost));
    out[hy::MLP_NPARAM + 2 * hy::MLP_IN] = h->margin;
    out[hy::MLP_NPARAM + 2 * hy::MLP_IN + 1] = (float)h->model_P;
    return HY_OK;
}

int hy_index_set_probe_model(hy_index* h, const float* in) {
    HY_CHECK(h && in, HY_ERR_ARG, "set_probe_model: NULL argument");
    h->epoch++;  // a captured search graph no longer matches
    HY_RET(set_device(h));
    HY_RET(h->m_params.ensure(hy::MLP_NPARAM * sizeof(float)));
    HY_RET(h->m_mu.ensure(hy::MLP_IN * sizeof(float)));
    HY_RET(h->m_sd.ensure(hy::MLP_IN * sizeof(float)));
    HY_CUDA(cudaMemcpy(h->m_params.p, in, hy::MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    HY_CUDA(cudaMemcpy(h->m_mu.p, in + hy::MLP_NPARAM, hy::MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    HY_CUDA(cudaMemcpy(h->m_sd.p, in + hy::MLP_NPARAM + hy::MLP_IN, hy::MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    h->margin = in[hy::MLP_NPARAM + 2 * hy::MLP_IN];
    h->model_P = (int)in[hy::MLP_NPARAM + 2 * hy::MLP_IN + 1];
    h->learned_mean = 0;
    HY_RET(h->m_wimg.ensure(hy::mlp_wimg_bytes()));
    HY_CUDA(hy::mlp_pack(h->m_params.as<float>(), h->m_wimg.as<unsigned char>(), nullptr));
    HY_CUDA(cudaDeviceSynchronize());
    h->model_ready = true;
    return HY_OK;
}

int hy_index_search_preassigned(hy_index* h, size_t n, const float* q, size_t k, size_t nprobe, const int64_t* probes,
                                float* D, int64_t* I) {
    HY_CHECK(h && (n == 0 || (q && probes && D && I)), HY_ERR_ARG, "search_preassigned: NULL argument");
    std::lock_guard<std::mutex> g(h->mu);
    if (n == 0) return HY_OK;
    HY_RET(check_search_args(h, n, k));
    HY_CHECK(nprobe >= 1, HY_ERR_ARG, "search_preassigned: nprobe must be >= 1");
    for (size_t i = 0; i < n * nprobe; ++i)
        HY_CHECK(probes[i] >= -1 && probes[i] < (int64_t)h->nlist, HY_ERR_ARG, "search_preassigned: list id out of range");
    HY_RET(set_device(h));
    cudaStream_t s = h->stream;
    HY_RET(h->w_q.ensure(n * h->d * sizeof(float)));
    HY_RET(h->w_probes.ensure(n * nprobe * sizeof(int64_t)));
    HY_RET(h->w_D.ensure(n * k * sizeof(float)));
    HY_RET(h->w_I.ensure(n * k * sizeof(int64_t)));
    HY_RET(reset_counters(h, s));
    HY_CUDA(cudaMemcpyAsync(h->w_q.p, q, n * h->d * sizeof(float), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemcpyAsync(h->w_probes.p, probes, n * nprobe * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    const uint32_t* thr = nullptr;
    if (h->warmup_list > 0 && h->metric == HY_METRIC_L2) {
        const size_t wls = h->warmup_list_size ? h->warmup_list_size : k;
        HY_CHECK(std::min(h->warmup_list, nprobe) * wls <= 32768, HY_ERR_ARG,
                 "presearch: warmup_list * warmup_list_size above 32768");
        HY_RET(h->w_thr.ensure(n * sizeof(uint32_t)));
        HY_CUDA(hy::launch_warmup(h->L, h->codes.as<float>(), h->list_off.as<int64_t>(), h->list_size.as<int32_t>(),
                                  h->w_q.as<float>(), (int)n, h->w_probes.as<int64_t>(), (int)nprobe, (int)k,
                                  (int)h->warmup_list, (int)wls, 1, h->w_thr.as<uint32_t>(), nullptr,
                                  h->w_err.as<int>(), s));
        thr = h->w_thr.as<uint32_t>();
    }
    h->ev = h->ev_direct;
    HY_CUDA(ev_record(h->ev[0], s));
    HY_CUDA(ev_record(h->ev[1], s));
    HY_RET(scan_and_merge(h, n, h->w_q.as<float>(), k, nprobe, h->w_probes.as<int64_t>(), thr, h->w_D.as<float>(),
                          h->w_I.as<int64_t>(), s, true));
    HY_CUDA(cudaMemcpyAsync(D, h->w_D.p, n * k * sizeof(float), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaMemcpyAsync(I, h->w_I.p, n * k * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    return finish_host_call(h, s, true, n, nprobe);
}

int hy_index_probes(hy_index* h, size_t n, const float* q, int64_t* probes) {
    HY_CHECK(h && (n == 0 || (q && probes)), HY_ERR_ARG, "probes: NULL argument");
    std::lock_guard<std::mutex> g(h->mu);
    if (n == 0) return HY_OK;
    HY_CHECK(h->trained, HY_ERR_STATE, "probes: index is not trained");
    HY_CHECK(h->nlist <= 40000, HY_ERR_ARG, "probes: nlist above 40000 is not supported by the coarse selector");
    HY_RET(set_device(h));
    cudaStream_t s = h->stream;
    const size_t nprobe = std::min(h->nprobe, h->nlist);
    const size_t qc = query_chunk(h->nlist, n);
    HY_RET(h->w_q.ensure(n * h->d * sizeof(float)));
    HY_RET(h->w_scores.ensure(qc * h->nlist * sizeof(float)));
    HY_RET(h->w_probes.ensure(n * nprobe * sizeof(int64_t)));
    if (learned_on(h)) {
        HY_RET(h->m_pscore.ensure(qc * nprobe * sizeof(float)));
        HY_RET(h->m_total.ensure(sizeof(unsigned long long)));
    }
    HY_CUDA(cudaMemcpyAsync(h->w_q.p, q, n * h->d * sizeof(float), cudaMemcpyHostToDevice, s));
    const bool tensor = coarse_on_tensor(h, nprobe);
    if (tensor) {
        HY_RET(ensure_common(h));
        if (h->nsm == 0) HY_CUDA(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
        HY_RET(h->b_qb.ensure(qc * ((h->d + 63) / 64) * 128));
        HY_RET(h->b_qn.ensure(qc * sizeof(float4)));
        HY_RET(h->b_thr.ensure(qc * sizeof(float)));
    }
    for (size_t q0 = 0; q0 < n; q0 += qc) {
        const size_t m = std::min(qc, n - q0);
        const float* qq = h->w_q.as<float>() + q0 * h->d;
        if (tensor) {
            HY_CUDA(hy::launch_prep_queries(qq, (int)m, (int)h->d, h->b_qb.p, h->b_qn.as<float4>(), nullptr, s));
            HY_RET(coarse_tensor(h, m, qq, nprobe, h->w_probes.as<int64_t>() + q0 * nprobe,
                                 learned_on(h) ? h->m_pscore.as<float>() : nullptr, s));
        } else {
            HY_CUDA(hy::launch_coarse_scores(qq, (int)m, h->cent.as<float>(), (int)h->nlist, (int)h->d, h->metric,
                                             h->w_scores.as<float>(), s));
            HY_CUDA(hy::launch_select(h->w_scores.as<float>(), (int)m, (int)h->nlist, (int)nprobe,
                                      h->w_probes.as<int64_t>() + q0 * nprobe,
                                      learned_on(h) ? h->m_pscore.as<float>() : nullptr, s));
        }
        if (learned_on(h)) HY_RET(apply_learned_probes(h, m, nprobe, s, h->w_probes.as<int64_t>() + q0 * nprobe));
    }
    HY_CUDA(cudaMemcpyAsync(probes, h->w_probes.p, n * nprobe * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaStreamSynchronize(s));
    return HY_OK;
}

int hy_index_warmup_tops(hy_index* h, size_t n, const float* q, size_t k, size_t nprobe, const int64_t* probes,
                         size_t warmup_list, size_t warmup_list_size, float* tops) {
    HY_CHECK(h && (n == 0 || (q && probes && tops)), HY_ERR_ARG, "warmup_tops: NULL argument");
    std::lock_guard<std::mutex> g(h->mu);
    if (n == 0) return HY_OK;
    HY_CHECK(k >= 1, HY_ERR_ARG, "warmup_tops: k must be >= 1");
    HY_CHECK(nprobe >= 1 && warmup_list >= 1, HY_ERR_ARG, "warmup_tops: nprobe and warmup_list must be >= 1");
    if (warmup_list_size == 0) warmup_list_size = k;
    HY_CHECK(std::min(warmup_list, nprobe) * warmup_list_size <= 32768, HY_ERR_ARG,
             "warmup_tops: warmup_list * warmup_list_size above 32768");
    for (size_t i = 0; i < n * nprobe; ++i)
        HY_CHECK(probes[i] >= -1 && probes[i] < (int64_t)h->nlist, HY_ERR_ARG, "warmup_tops: list id out of range");
    HY_CHECK(h->ntotal > 0 || h->arena_rows == 0, HY_ERR_STATE, "warmup_tops: no lists");
    HY_RET(set_device(h));
    cudaStream_t s = h->stream;
    HY_RET(ensure_common(h));
    HY_RET(h->w_q.ensure(n * h->d * sizeof(float)));
    HY_RET(h->w_probes.ensure(n * nprobe * sizeof(int64_t)));
    HY_RET(h->w_thr.ensure(n * sizeof(uint32_t)));
    HY_RET(h->w_f.ensure(n * sizeof(float)));
    HY_CUDA(cudaMemcpyAsync(h->w_q.p, q, n * h->d * sizeof(float), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemcpyAsync(h->w_probes.p, probes, n * nprobe * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    if (h->arena_rows == 0) {
        std::vector<float> mx(n, FLT_MAX);
        std::memcpy(tops, mx.data(), n * sizeof(float));
        return HY_OK;
    }
    HY_CUDA(hy::launch_warmup(h->L, h->codes.as<float>(), h->list_off.as<int64_t>(), h->list_size.as<int32_t>(),
                              h->w_q.as<float>(), (int)n, h->w_probes.as<int64_t>(), (int)nprobe, (int)k,
                              (int)warmup_list, (int)warmup_list_size, 0, h->w_thr.as<uint32_t>(), h->w_f.as<float>(),
                              h->w_err.as<int>(), s));
    HY_CUDA(cudaMemcpyAsync(tops, h->w_f.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    HY_CUDA(cudaStreamSynchronize(s));
    return HY_OK;
}

int hy_index_last_stats(const hy_index* hc, hy_search_stats_t* out) {
    HY_CHECK(hc && out, HY_ERR_ARG, "last_stats: NULL argument");
    hy_index* h = const_cast<hy_index*>(hc);
    if (h->times_pending) {
        // The device-API search returns before its kernels finish; its
        // device times are read here, once its last event has completed.
        std::lock_guard<std::mutex> g(h->mu);
        HY_RET(set_device(h));
        HY_CUDA(cudaEventSynchronize(h->ev[4]));
        collect_times(h);
        if ((batched_form(h) || h->lm_last) && h->b_fbtot.p) {
            unsigned long long c = 0;
            HY_CUDA(cudaMemcpy(&c, h->b_fbtot.p, sizeof(c), cudaMemcpyDeviceToHost));
            h->stats.fallback_queries = c;
        }
        if (h->w_counters.p) {
            unsigned long long c[4] = {0, 0, 0, 0};
            HY_CUDA(cudaMemcpy(c, h->w_counters.p, sizeof(c), cudaMemcpyDeviceToHost));
            h->stats.tile_blocks = c[0];
            h->stats.tile_blocks_max = c[1];
            h->stats.seg_sums = c[2];
            h->stats.seg_sums_max = c[3];
        }
    }
    *out = h->stats;
    return HY_OK;
}

int hy_index_list_size(const hy_index* h, size_t list, size_t* size) {
    HY_CHECK(h && size, HY_ERR_ARG, "list_size: NULL argument");
    HY_CHECK(list < h->nlist, HY_ERR_ARG, "list_size: list id out of range");
    *size = h->h_list_size.empty() ? 0 : (size_t)h->h_list_size[list];
    return HY_OK;
}

int hy_index_get_list(const hy_index* hc, size_t list, int64_t* ids, float* codes, float* norms) {
    HY_CHECK(hc, HY_ERR_ARG, "get_list: NULL handle");
    HY_CHECK(list < hc->nlist, HY_ERR_ARG, "get_list: list id out of range");
    hy_index* h = const_cast<hy_index*>(hc);
    std::lock_guard<std::mutex> g(h->mu);
    if (h->h_list_size.empty() || h->h_list_size[list] == 0) return HY_OK;
    HY_RET(set_device(h));
    const int n = h->h_list_size[list];
    const int64_t r0 = h->h_list_off[list];
    cudaStream_t s = h->stream;
    if (ids) HY_CUDA(cudaMemcpyAsync(ids, h->ids.as<int64_t>() + r0, n * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    if (norms) HY_CUDA(cudaMemcpyAsync(norms, h->norms.as<float>() + r0, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (codes) {
        HY_RET(h->w_f.ensure((size_t)n * h->d * sizeof(float)));
        HY_CUDA(hy::launch_unpack_list(h->L, h->codes.as<float>(), r0, n, h->w_f.as<float>(), s));
        HY_CUDA(cudaMemcpyAsync(codes, h->w_f.p, (size_t)n * h->d * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    HY_CUDA(cudaStreamSynchronize(s));
    return HY_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Read-only view of an index's device data for entry points defined in other
// files of the library (hy_noalloc.cu).
namespace hy {
struct IndexView {
    ArenaLayout L;
    const float* codes;
    const int64_t* list_off;
    const int32_t* list_size;
    const int64_t* ids;
    int metric;
    size_t d, nlist;
    int device;
    bool trained, has_lists;
};
int index_view(const hy_index* h, IndexView* v) {
    if (!h || !v) return fail(HY_ERR_ARG, "index_view: NULL argument");
    v->L = h->L;
    v->codes = h->codes.as<float>();
    v->list_off = h->list_off.as<int64_t>();
    v->list_size = h->list_size.as<int32_t>();
    v->ids = h->ids.as<int64_t>();
    v->metric = h->metric;
    v->d = h->d;
    v->nlist = h->nlist;
    v->device = h->device;
    v->trained = h->trained;
    v->has_lists = !h->h_list_size.empty();
    return HY_OK;
}
int set_error(int code, const char* msg) { return fail(code, msg); }
// The index's call lock: an entry point that reads the index's device data
// across several launches holds it until its last launch has completed, so
// a concurrent add / load / reset cannot free that data under it.
std::mutex& index_mutex(hy_index* h) { return h->mu; }
}  // namespace hy

// ---------------------------------------------------------------------------
// The reference's .index format (src/Index.cpp:1708-1770, src/IVF.cpp:76-134):
//   size_t d, size_t nlist, int32 metric, int32 opt_level, size_t sub_k,
//   size_t sub_nlist, size_t sub_nprobe, float centroids[nlist*d], then for
//   each non-empty list: size_t list_id, size_t list_size, size_t d,
//   size_t sub_k, int32 opt_level, size_t ids[list_size],
//   float codes[list_size*d], float norms[list_size], and the optional
//   arrays its opt_level carries (skipped on load, never written).
namespace {

struct FileList {
    size_t id = 0;
    std::vector<int64_t> ids;
    std::vector<float> codes;
};

struct FileIndex {
    size_t d = 0, nlist = 0, sub_k = 0, sub_nlist = 1, sub_nprobe = 1;
    int32_t metric = 1, opt_level = 0;
    std::vector<float> cent;
    std::vector<FileList> lists;
};

template <class T>
bool rd(std::ifstream& in, T* v, size_t n = 1) {
    in.read(reinterpret_cast<char*>(v), static_cast<std::streamsize>(sizeof(T) * n));
    return static_cast<bool>(in);
}

int read_index_file(const char* path, FileIndex* f, bool with_data) {
    std::ifstream in(path, std::ios::binary);
    HY_CHECK(in.is_open(), HY_ERR_IO, std::string("cannot open file ") + path);
    HY_CHECK(rd(in, &f->d) && rd(in, &f->nlist) && rd(in, &f->metric) && rd(in, &f->opt_level) && rd(in, &f->sub_k) &&
                 rd(in, &f->sub_nlist) && rd(in, &f->sub_nprobe),
             HY_ERR_IO, "truncated .index header");
    HY_CHECK(f->d >= 1 && f->d <= 4096 && f->nlist >= 1 && f->nlist <= (size_t(1) << 24), HY_ERR_IO,
             "corrupt .index header (d or nlist out of range)");
    HY_CHECK(f->metric == 0 || f->metric == 1, HY_ERR_IO, "corrupt .index header (metric)");
    f->cent.resize(f->nlist * f->d);
    HY_CHECK(rd(in, f->cent.data(), f->cent.size()), HY_ERR_IO, "truncated .index centroids");
    for (;;) {
        size_t lid;
        in.read(reinterpret_cast<char*>(&lid), sizeof(lid));
        if (in.eof() && in.gcount() == 0) break;
        HY_CHECK(in.gcount() == sizeof(lid), HY_ERR_IO, "truncated .index list header");
        HY_CHECK(lid < f->nlist, HY_ERR_IO, "corrupt .index list id");
        size_t n, d, subk;
        int32_t opt;
        HY_CHECK(rd(in, &n) && rd(in, &d) && rd(in, &subk) && rd(in, &opt), HY_ERR_IO, "truncated .index list header");
        HY_CHECK(d == f->d && n < (size_t(1) << 31), HY_ERR_IO, "corrupt .index list (dimension or size)");
        FileList L;
        L.id = lid;
        std::vector<uint64_t> ids(n);
        HY_CHECK(rd(in, ids.data(), n), HY_ERR_IO, "truncated .index list ids");
        std::vector<float> codes;
        if (with_data) {
            codes.resize(n * d);
            HY_CHECK(rd(in, codes.data(), n * d), HY_ERR_IO, "truncated .index list codes");
        } else {
            in.seekg(static_cast<std::streamoff>(n * d * sizeof(float)), std::ios::cur);
        }
        size_t skip = n * sizeof(float);  // norms (recomputed on load)
        if ((opt & 1) || (opt & 4)) skip += 2 * n * sizeof(float);
        if (opt & 2) skip += n * subk * (sizeof(int64_t) + sizeof(float));
        if (opt & 4) skip += 2 * n * subk * (sizeof(int64_t) + sizeof(float));
        in.seekg(static_cast<std::streamoff>(skip), std::ios::cur);
        HY_CHECK(static_cast<bool>(in), HY_ERR_IO, "truncated .index list payload");
        L.ids.assign(ids.begin(), ids.end());
        L.codes = std::move(codes);
        f->lists.push_back(std::move(L));
    }
    return HY_OK;
}

}  // namespace

extern "C" {

int hy_file_inspect(const char* path, size_t* d, size_t* nlist, int* metric, int* opt_level, size_t* nonempty_lists,
                    size_t* ntotal) {
    HY_CHECK(path, HY_ERR_ARG, "file_inspect: NULL path");
    FileIndex f;
    HY_RET(read_index_file(path, &f, false));
    size_t tot = 0;
    for (auto& l : f.lists) tot += l.ids.size();
    if (d) *d = f.d;
    if (nlist) *nlist = f.nlist;
    if (metric) *metric = f.metric;
    if (opt_level) *opt_level = f.opt_level;
    if (nonempty_lists) *nonempty_lists = f.lists.size();
    if (ntotal) *ntotal = tot;
    return HY_OK;
}

int hy_index_save(const hy_index* hc, const char* path) {
    HY_CHECK(hc && path, HY_ERR_ARG, "save: NULL argument");
    HY_CHECK(hc->trained, HY_ERR_STATE, "save: index is not trained");
    hy_index* h = const_cast<hy_index*>(hc);
    std::ofstream out(path, std::ios::binary);
    HY_CHECK(out.is_open(), HY_ERR_IO, std::string("Cannot open file ") + path);
    auto wr = [&](const void* p, size_t bytes) { out.write(static_cast<const char*>(p), static_cast<std::streamsize>(bytes)); };
    const int32_t metric = h->metric, opt = 0;
    wr(&h->d, sizeof(size_t));
    wr(&h->nlist, sizeof(size_t));
    wr(&metric, 4);
    wr(&opt, 4);
    wr(&h->sub_k, sizeof(size_t));
    wr(&h->sub_nlist, sizeof(size_t));
    wr(&h->sub_nprobe, sizeof(size_t));
    wr(h->h_cent.data(), h->nlist * h->d * sizeof(float));
    for (size_t l = 0; l < h->nlist && !h->h_list_size.empty(); ++l) {
        const size_t n = (size_t)h->h_list_size[l];
        if (n == 0) continue;
        std::vector<int64_t> ids(n);
        std::vector<float> codes(n * h->d), norms(n);
        HY_RET(hy_index_get_list(h, l, ids.data(), codes.data(), norms.data()));
        // The reference fills candidate_norms only for L2 (src/Index.cpp:689-696).
        if (h->metric != HY_METRIC_L2) std::fill(norms.begin(), norms.end(), 0.0f);
        const size_t subk = 0;
        std::vector<uint64_t> uids(ids.begin(), ids.end());
        wr(&l, sizeof(size_t));
        wr(&n, sizeof(size_t));
        wr(&h->d, sizeof(size_t));
        wr(&subk, sizeof(size_t));
        wr(&opt, 4);
        wr(uids.data(), n * sizeof(uint64_t));
        wr(codes.data(), n * h->d * sizeof(float));
        wr(norms.data(), n * sizeof(float));
    }
    HY_CHECK(static_cast<bool>(out), HY_ERR_IO, std::string("write failed: ") + path);
    return HY_OK;
}

int hy_index_load(hy_index* h, const char* path) {
    HY_CHECK(h && path, HY_ERR_ARG, "load: NULL argument");
    h->epoch++;  // a captured search graph no longer matches
    FileIndex f;
    HY_RET(read_index_file(path, &f, true));
    std::lock_guard<std::mutex> g(h->mu);
    HY_RET(set_device(h));
    cudaStream_t s = h->stream;
    h->d = f.d;
    h->nlist = f.nlist;
    h->metric = f.metric;
    h->sub_k = f.sub_k;
    h->sub_nlist = f.sub_nlist;
    h->sub_nprobe = f.sub_nprobe;
    h->opt_level = 0;  // load_index resets opt_level (src/Index.cpp:1746)
    h->dim_blocks = std::min<size_t>(h->dim_blocks ? h->dim_blocks : 4, h->d);
    h->L = make_layout((int)h->d, (int)h->dim_blocks);
    HY_RET(h->cent.ensure(h->nlist * h->d * sizeof(float)));
    h->h_cent = f.cent;
    HY_CUDA(cudaMemcpyAsync(h->cent.p, h->h_cent.data(), h->nlist * h->d * sizeof(float), cudaMemcpyHostToDevice, s));
    h->trained = true;
    h->cimg_valid = false;
    // Rows list by list in file order; a later record of the same list
    // replaces an earlier one, as load_IVF does.
    std::vector<const FileList*> byid(h->nlist, nullptr);
    for (auto& l : f.lists) byid[l.id] = &l;
    std::vector<int32_t> sizes(h->nlist, 0);
    size_t n = 0;
    for (size_t l = 0; l < h->nlist; ++l)
        if (byid[l]) {
            sizes[l] = (int32_t)byid[l]->ids.size();
            n += byid[l]->ids.size();
        }
    std::vector<float> rows(std::max<size_t>(n, 1) * h->d);
    std::vector<int64_t> labels(std::max<size_t>(n, 1)), srcid(std::max<size_t>(n, 1));
    std::vector<int32_t> order(std::max<size_t>(n, 1));
    size_t p = 0;
    for (size_t l = 0; l < h->nlist; ++l) {
        if (!byid[l]) continue;
        const FileList& L = *byid[l];
        std::memcpy(&rows[p * h->d], L.codes.data(), L.codes.size() * sizeof(float));
        for (size_t i = 0; i < L.ids.size(); ++i) {
            labels[p + i] = (int64_t)l;
            srcid[p + i] = L.ids[i];
            order[p + i] = (int32_t)(p + i);
        }
        p += L.ids.size();
    }
    HY_RET(h->w_x.ensure(rows.size() * sizeof(float)));
    HY_RET(h->w_lab.ensure(labels.size() * sizeof(int64_t)));
    HY_RET(h->w_vals2.ensure(order.size() * sizeof(int32_t)));
    HY_CUDA(cudaMemcpyAsync(h->w_x.p, rows.data(), rows.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemcpyAsync(h->w_lab.p, labels.data(), labels.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    HY_CUDA(cudaMemcpyAsync(h->w_vals2.p, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    HY_RET(build_arena(h, h->w_x.as<float>(), n, h->w_vals2.as<int32_t>(), h->w_lab.as<int64_t>(), sizes, s));
    // build_arena stored the row position as the id; restore the file's ids.
    std::vector<int64_t> arena_ids(std::max<size_t>(h->arena_rows, 32), -1);
    p = 0;
    for (size_t l = 0; l < h->nlist; ++l) {
        for (int32_t i = 0; i < sizes[l]; ++i) arena_ids[h->h_list_off[l] + i] = srcid[p + i];
        p += sizes[l];
    }
    HY_CUDA(cudaMemcpy(h->ids.p, arena_ids.data(), arena_ids.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
    return HY_OK;
}

}  // extern "C"
