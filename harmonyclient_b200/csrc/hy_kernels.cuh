// Host-visible declarations of the IVF kernels' launchers (hy_kernels.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "hy_device.cuh"

namespace hy {

// Layout of the list arena (device).  Rows are grouped in tiles of 32; each
// list starts on a tile boundary and its tail is padded with zero rows whose
// id is -1.  Inside a tile, the dimensions are split into `nb` blocks; block b
// of all 32 rows is one contiguous run of 32 * pitch[b] floats, so the rows'
// block b is a single bulk copy and a tile whose rows are all pruned after
// block b never loads blocks b+1...  Within a row's block, 16-byte chunk c is
// stored at chunk (c & ~7) | ((c ^ row) & 7), which lets 32 lanes reading the
// same logical chunk of 32 rows hit 32 different shared-memory banks.
struct ArenaLayout {
    int d = 0;
    int nb = 0;                        // dimension blocks
    int bstart[MAX_BLOCKS + 1] = {};   // first dimension of block b (bstart[nb] = d)
    int pitch[MAX_BLOCKS] = {};        // floats per row of block b (multiple of 32)
    int boff[MAX_BLOCKS + 1] = {};     // float offset of block b inside a row
    int row_pitch = 0;                 // boff[nb]
    int max_pitch = 0;
};

// Float offset of (arena row r, block b, dimension j within the block).
__host__ __device__ inline size_t arena_offset(const ArenaLayout& L, int64_t r, int b, int j) {
    const int64_t tile = r >> 5;
    const int lr = static_cast<int>(r & 31);
    const int c = j >> 2;
    const int pc = (c & ~7) | ((c ^ lr) & 7);
    return static_cast<size_t>(tile) * 32 * L.row_pitch + static_cast<size_t>(L.boff[b]) * 32 +
           static_cast<size_t>(lr) * L.pitch[b] + static_cast<size_t>(pc) * 4 + (j & 3);
}

struct ScanParams {
    ArenaLayout L;
    const float* codes;        // arena
    const int64_t* list_off;   // [nlist+1] first arena row of each list
    const int32_t* list_size;  // [nlist] rows in each list
    const float* q;            // [nq][d]
    const int64_t* probes;     // [nq][nprobe], -1 = skip
    const uint32_t* init_thr;  // [nq] ordered-key thresholds or nullptr
    uint32_t* g_thr;           // [nq] shared threshold across splits or nullptr
    uint64_t* out;             // [nq][nsplit][KR*32] sorted keys
    unsigned long long* counters;  // [2]: tile blocks loaded, tile blocks possible
    int* err;
    int nq, nprobe, nsplit, k, metric, prune;
    const int32_t* nq_dev = nullptr;  // optional device count: queries at or past it are skipped
    // With nq_dev: the launch has min(nq, qgrid) query slots (qgrid > 0) whose
    // CTAs loop over the queries below the device count.
    int qgrid = 0;
};

cudaError_t launch_coarse_scores(const float* q, int nq, const float* cent, int nlist, int d, int metric, float* out,
                                 cudaStream_t s);
cudaError_t launch_select(const float* scores, int nq, int n, int m, int64_t* out_idx, float* out_score,
                          cudaStream_t s);
cudaError_t launch_argmin(const float* scores, int nrows, int n, int64_t* out_idx, float* out_score,
                          cudaStream_t s);
// skip_lo <= skip_hi: a query whose nearest list has between skip_lo and
// skip_hi rows gets no warm-up (threshold FLT_MAX); the batched search's dense
// first pass bounds it instead.
cudaError_t launch_warmup(const ArenaLayout& L, const float* codes, const int64_t* list_off,
                          const int32_t* list_size, const float* q, int nq, const int64_t* probes, int nprobe, int k,
                          int wl, int wls, int blockwise, uint32_t* out_thr, float* out_f, int* err, cudaStream_t s,
                          int skip_lo = 0, int skip_hi = -1);
cudaError_t launch_scan_plain(const ScanParams& p, int* smem_bytes_out, cudaStream_t s);
// rows (optional): the arena row of every result (-1 when unfilled).
// nq_dev (optional): device count; queries at or past it are skipped.
cudaError_t launch_merge(const uint64_t* parts, int nq, int nparts, int kp, int k, int metric, const int64_t* ids,
                         float* D, int64_t* I, cudaStream_t s, int64_t* rows = nullptr,
                         const int32_t* nq_dev = nullptr);

// Per-query nprobe: probes at or beyond np[q] (clamped to [1, P]) become -1.
cudaError_t launch_cut_probes(int64_t* probes, int n, int P, const int32_t* np, cudaStream_t s);

// Learned probe predictor helpers (see hy_kernels.cu).
cudaError_t launch_probe_features(const float* scores, int n, int P, const float* mu, const float* sd, float* X,
                                  cudaStream_t s);
cudaError_t launch_stop_labels(const int64_t* rows, int n, int kl, const int64_t* probes, int P,
                               const int64_t* list_off, int nlist, float* label, cudaStream_t s);
cudaError_t launch_apply_nprobe(const float* y, int n, float margin, int P, int64_t* probes,
                                unsigned long long* total, cudaStream_t s);

// Index construction.
cudaError_t launch_histogram(const int64_t* labels, int64_t n, int32_t* counts, cudaStream_t s);
cudaError_t launch_make_sort_keys(const int64_t* labels, const float* score, int64_t n, uint64_t* keys,
                                  int32_t* vals, cudaStream_t s);
cudaError_t radix_sort_pairs(void* tmp, size_t* tmp_bytes, const uint64_t* kin, uint64_t* kout, const int32_t* vin,
                             int32_t* vout, int64_t n, int end_bit, cudaStream_t s);
// Merge of parts per-query top-k lists ([parts][n][k], best first) into the
// best k (ties: part order, then rank).
cudaError_t launch_merge_parts(const float* D, const int64_t* I, int parts, int n, int k, int metric, float* oD,
                               int64_t* oI, cudaStream_t s);
// keep (optional): rows of list l past keep[l] are not stored (lists an index
// does not hold have keep 0).
cudaError_t launch_scatter(const ArenaLayout& L, const float* x, int64_t n, const int32_t* order,
                           const int64_t* labels, const int64_t* list_start, const int64_t* list_off,
                           const int32_t* keep, float* codes, int64_t* ids, float* norms, cudaStream_t s);
cudaError_t launch_fill_i64(int64_t* p, int64_t n, int64_t v, cudaStream_t s);
cudaError_t launch_gather_rows(const float* x, const int64_t* rows, int64_t n, int d, float* out, cudaStream_t s);
cudaError_t launch_normalize_rows(const float* x, int64_t n, int d, float* out, cudaStream_t s);
cudaError_t launch_kmeans_accumulate(const float* x, const int64_t* labels, int64_t n, int d, double* sums,
                                     unsigned long long* counts, cudaStream_t s);
cudaError_t launch_kmeans_update(const double* sums, const unsigned long long* counts, int nlist, int d,
                                 float* cent, cudaStream_t s);
cudaError_t launch_normalize_centroids(float* cent, int nlist, int d, cudaStream_t s);
cudaError_t launch_unpack_list(const ArenaLayout& L, const float* codes, int64_t row0, int n, float* out,
                               cudaStream_t s);

}  // namespace hy
