// Host-visible launchers of the batched tensor-core scan (hy_batched.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hy_kernels.cuh"

namespace hy {

constexpr int BATCH_ROW_ALIGN = 128;  // lists start on 128-row tiles
constexpr int BATCH_KB_BYTES = 16384;  // one k-block (128 rows x 64 bf16)

// Bytes of the bf16 tensor-core image of an arena of `rows` rows (multiple of
// 128) and dimension d.
inline size_t bf16_image_bytes(int64_t rows, int d) {
    const int nkb = (d + 63) / 64;
    return static_cast<size_t>(rows / BATCH_ROW_ALIGN) * nkb * BATCH_KB_BYTES;
}
// The split (hi, lo) bf16 image of launch_centroid_image.
inline size_t bf16_split_image_bytes(int64_t rows, int d) { return 2 * bf16_image_bytes(rows, d); }

// Bytes of the e4m3 image (128-byte k-blocks of 128 dimensions).
inline size_t f8_image_bytes(int64_t rows, int d) {
    const int nkb = (d + 127) / 128;
    return static_cast<size_t>(rows / BATCH_ROW_ALIGN) * nkb * BATCH_KB_BYTES;
}

// Queries per group of the batched kernel for dimension d (128, 64 or 32:
// the largest whose shared-memory footprint fits), 0 if none fits.
int batched_group_size(int d, bool f8);

cudaError_t launch_to_bf16_arena(const ArenaLayout& L, const float* codes, int64_t rows, void* out, cudaStream_t s);
// e4m3 image with per-list scales: tile_max [rows/128] scratch, lscale
// [nlist] and tscale [rows/128] outputs.
cudaError_t launch_to_f8_arena(const ArenaLayout& L, const float* codes, int64_t rows, const int64_t* list_off,
                               const int32_t* list_size, int nlist, float* tile_max, float* lscale, float* tscale,
                               void* out, cudaStream_t s);
// qscale == nullptr: bf16 queries; else e4m3 queries with per-query scales.
// bf16 queries with qexact: qexact[i] = 1 when query i and the arena admit
// exact tensor-core distances: amax >= 0 (the arena's certificate, see
// launch_arena_integral: every value an integer of magnitude <= 256 and the
// largest row squared norm amax), the query's values integers of magnitude
// <= 256 and |q|^2 + amax < 2^23.  Then every product and partial sum of the
// bf16 distance is an integer below 2^24, exact in f32, and the distance
// equals the plain scan's bit for bit.
cudaError_t launch_prep_queries(const float* q, int nq, int d, void* qb, float4* qaux, float* qscale, cudaStream_t s,
                                float amax = -1.0f, int32_t* qexact = nullptr);
// flag (int, preset to 1) := 0 unless every one of the n values of codes is
// an integer of magnitude <= 256; maxxn (preset to 0) := bit pattern of the
// largest of xn[0..rows).
cudaError_t launch_arena_integral(const float* codes, int64_t n, const float* xn, int64_t rows, int* flag,
                                  unsigned int* maxxn, cudaStream_t s);
// Per arena row {|x~|, |x - x~|} for the error bound (tscale == nullptr: the
// bf16 image, else the e4m3 image with those tile scales), and per 128-row
// tile the maxima of both.
// tile_max[t] = the largest xn over rows [128 t, 128 t + 128) (rows a
// multiple of 128).
cudaError_t launch_tile_max(const float* xn, int64_t rows, float* tile_max, cudaStream_t s);
cudaError_t launch_row_aux(const ArenaLayout& L, const float* codes, int64_t rows, const float* tscale, float2* aux,
                           float2* tile_aux, cudaStream_t s);

// Work buffers of one batched search.
struct BatchWork {
    int32_t* pair_cnt;   // [nlist]
    int32_t* pair_fill;  // [nlist]
    int64_t* pair_off;   // [nlist+1]
    int32_t* pairs;      // [nq*nprobe]
    int32_t* item_cnt;   // [nlist]
    int64_t* item_off;   // [nlist+1]
    int4* items;         // [item_cap] item descriptors
    int64_t item_cap;
    unsigned int* work;  // [1]
    uint64_t* cand;      // [nq*capq]
    int32_t* cand_cnt;   // [nq]
    int32_t* overflow;   // [1 + nq]: count, then query ids
    int32_t* big;        // [1 + nq]: queries re-ranked by the CTA kernel (count, then ids)
    int32_t* big2;       // [1 + nq]: queries tightened by the CTA kernel (count, then ids)
    int32_t* rest = nullptr;  // [1 + nq]: queries whose first-pass list was not dense (count, then ids)
    unsigned int* done = nullptr;  // [1], zero between launches: the inversion's ticket
};

// Inverts probe columns [j0, j1) of every query into per-list query groups
// and builds the work items.
cudaError_t launch_invert_probes(const int64_t* probes, int nq, int nprobe, int j0, int j1, int nlist,
                                 const int32_t* list_size, int rs, int qg, const BatchWork& w, cudaStream_t s);
// The first pass's dense lists: a query whose probes[q * nprobe] list has at
// most dense_max rows (capped at capq) holds one f32 score per row of that
// list in the upper half of its buffer (bytes 4 capq + 4 i).  dense_max 0:
// no dense lists.
struct DenseFirst {
    const int64_t* probes = nullptr;
    int nprobe = 0;
    const int32_t* list_size = nullptr;
    const int64_t* list_off = nullptr;
    int dense_max = 0;
    const float2* tile_aux = nullptr;  // per arena tile {max |x~|, max |x - x~|}
    const float* tile_xn = nullptr;    // per arena tile, max |x|^2
};
// thr := min(thr, k-th smallest upper bound over each query's candidates),
// and the candidates that can still reach the top-k are compacted as keys.
cudaError_t launch_tighten(const float* xn, const float2* xaux, const float4* qaux, int nq, const BatchWork& w,
                           int capq, int k, int metric, int d, bool f8, int nsm, float* thr, cudaStream_t s,
                           DenseFirst df);

// The coarse quantiser on the tensor cores (bf16 form).  The centroids
// (row-major, nlist x d) as a one-list index: split bf16 image (per 64
// dimensions a hi k-block, bf16(c), then a lo k-block, bf16(c - hi); launched
// with BatchedLaunch::ksplit), per-row {|(|hi| + |lo|)|, |c - hi - lo|},
// per-tile maxima and squared norms, rows padded to whole 128-row tiles
// (img: bf16_split_image_bytes(rows), aux/xn: rows, tile_aux: rows/128).
cudaError_t launch_centroid_image(const float* cent, int nlist, int d, void* img, float2* aux, float2* tile_aux,
                                  float* xn, cudaStream_t s);
// Work of one coarse launch over nq queries: list_off[2], list_size[1] of the
// centroid index; w.pairs [nq], w.items [ngroups*nslices], w.pair_cnt [1],
// w.pair_off [2], w.item_off [2].
cudaError_t launch_coarse_items(int nq, int nlist, int ngroups, int nslices, int64_t* list_off, int32_t* list_size,
                                const BatchWork& w, cudaStream_t s);
// From the dense scores of the coarse launch (cand, nq x nlist slots of 8
// bytes, scores in each query's upper half) and the bounds recomputed from
// cxn / caux (the centroid index's squared norms and {|c~|, |c - c~|}) and
// qaux: the exact m best centroids per query and their exact coarse scores,
// as launch_select gives them from coarse_scores (cand is overwritten).
// Needs m <= 256 and coarse_refine_smem(nlist, d, 1) <= 200 KiB.  A staging
// copy that does not complete within the wait limit raises *err.
size_t coarse_refine_smem(int nlist, int d, int warps);
cudaError_t launch_coarse_refine(float2* cand, int nq, int nlist, const float* q, const float* cent,
                                 const float* cxn, const float2* caux, const float4* qaux, int d, int metric, int m,
                                 int64_t* out_idx, float* out_score, int* err, cudaStream_t s);

// More than 2048 centroids: thr[q] := a bound on the m-th smallest
// score + bound among the S <= 1024 dense scores of query q (cand, nq x S
// slots, bounds recomputed as for launch_coarse_refine), then, from the keys
// a thresholded launch over all centroids emitted (cand + q * stride, ccnt[q]
// of them), the exact m best as launch_coarse_refine gives them (cand is
// overwritten).  cxn / caux: the centroid index's squared norms and
// {|c~|, |c - c~|}.
cudaError_t launch_coarse_thr(const float2* cand, int nq, int S, int m, const float* cxn, const float2* caux,
                              const float4* qaux, int d, int metric, float* thr, cudaStream_t s);
cudaError_t launch_coarse_refine_keys(uint64_t* cand, const int32_t* ccnt, int nq, int stride, const float* q,
                                      const float* cent, const float* cxn, const float2* caux, const float4* qaux,
                                      int d, int metric, int m, int64_t* out_idx, float* out_score, int* err,
                                      cudaStream_t s);

// Largest list the batched search's first pass scans densely (the candidate
// buffer's size caps it further).
constexpr size_t DENSE_MAX = 16384;

struct BatchedLaunch {
    const void* abf;
    const int64_t* list_off;
    const int32_t* list_size;
    const float* xn;
    const float2* tile_aux;
    const float2* xaux;  // per-row {|x~|, |x - x~|} of the operand type's image
    const void* qb;
    const float4* qaux;
    const float* thr;
    const float* lscale = nullptr;  // e4m3 form: per-list scales
    const float* qscale = nullptr;  // e4m3 form: per-query scales
    int nlist, d, rs, capq, metric, nsm;
    int qg = 128;     // queries per group (batched_group_size)
    bool f8 = false;  // e4m3 operands
    bool ksplit = false;  // abf is a split image (launch_centroid_image): two k-blocks per query k-block
    // Lists of at most dense_max rows (capped at capq) are scanned densely:
    // every row's f32 score lands at the row's offset in the list within the
    // upper half of the query's candidate buffer, with no threshold test, and the
    // query's count is set to the list size (each query must have one such
    // list in the launch; launch_tighten turns them into keys).  0 = every
    // list through the threshold test.
    int dense_max = 0;
};

cudaError_t launch_batched_scan(const BatchedLaunch& b, const BatchWork& w, int* err, cudaStream_t s);

// qbase: added to the query ids listed in w.overflow.  rmax > 0: at most the
// rmax candidates with the smallest tensor-core distance are re-ranked (the
// e4m3 form's oversampled re-rank); 0 re-ranks every candidate whose bound
// can reach the top-k.  qexact (optional, see launch_prep_queries): queries
// whose tensor-core distances are exact keep them instead of recomputing.
cudaError_t launch_rerank(const ArenaLayout& L, const float* codes, const int64_t* ids, const float* xn,
                          const float2* xaux, const float4* qaux, const float* q, int nq, const BatchWork& w, int qbase,
                          int capq, int k, int rmax, int metric, bool f8, int nsm, float* D, int64_t* I,
                          cudaStream_t s, const int32_t* qexact = nullptr);
cudaError_t launch_fill_f32(float* p, int64_t n, float v, cudaStream_t s);

// Device-side exact fallback for queries whose candidates overflowed
// (w.overflow: count, then chunk-local query ids).  Gather packs them
// (vectors and probe rows) to the front of fq / fprobes; scatter writes their
// plain-scan results back into D / I and adds the count to *total.  `cap` is
// the chunk's query count, so every overflowed query of the chunk fits.
cudaError_t launch_fb_gather(const int32_t* ovf, const float* q, const int64_t* probes, int nprobe, int d, int cap,
                             float* fq, int64_t* fprobes, int32_t* fcount, cudaStream_t s);
cudaError_t launch_fb_scatter(const int32_t* ovf, const float* fD, const int64_t* fI, int k, int cap, float* D,
                              int64_t* I, unsigned long long* total, cudaStream_t s);

}  // namespace hy
