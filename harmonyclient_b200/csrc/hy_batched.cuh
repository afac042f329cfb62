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

cudaError_t launch_to_bf16_arena(const ArenaLayout& L, const float* codes, int64_t rows, void* out, cudaStream_t s);
cudaError_t launch_prep_queries(const float* q, int nq, int d, void* qb, float4* qaux, cudaStream_t s);
// Per arena row {|x~|, |x - x~|} for the bf16 error bound, and per 128-row
// tile the maxima of both.
cudaError_t launch_row_aux(const ArenaLayout& L, const float* codes, int64_t rows, float2* aux, float2* tile_aux,
                           cudaStream_t s);

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
};

// Inverts probe columns [j0, j1) of every query into per-list query groups
// and builds the work items.
cudaError_t launch_invert_probes(const int64_t* probes, int nq, int nprobe, int j0, int j1, int nlist,
                                 const int32_t* list_size, int rs, const BatchWork& w, cudaStream_t s);
// thr := min(thr, k-th smallest upper bound over each query's candidates).
cudaError_t launch_tighten(const float* xn, const float2* xaux, const float4* qaux, int nq, const BatchWork& w,
                           int capq, int k, int metric, int d, float* thr, cudaStream_t s);

struct BatchedLaunch {
    const void* abf;
    const int64_t* list_off;
    const int32_t* list_size;
    const float* xn;
    const float2* tile_aux;
    const void* qb;
    const float4* qaux;
    const float* thr;
    int nlist, d, rs, capq, metric, nsm;
};

cudaError_t launch_batched_scan(const BatchedLaunch& b, const BatchWork& w, int* err, cudaStream_t s);

// qbase: global index of the chunk's first query (overflow ids are global).
cudaError_t launch_rerank(const ArenaLayout& L, const float* codes, const int64_t* ids, const float* xn,
                          const float2* xaux, const float4* qaux, const float* q, int nq, const BatchWork& w, int qbase,
                          int capq, int k, int metric, float* D, int64_t* I, cudaStream_t s);
cudaError_t launch_fill_f32(float* p, int64_t n, float v, cudaStream_t s);

// Device-side exact fallback for queries whose candidates overflowed
// (w.overflow: count, then chunk-local query ids).  Gather packs the first
// `cap` of them (vectors and probe rows) to the front of fq / fprobes;
// scatter writes their plain-scan results back into D / I and adds the count
// to *total (and the ones beyond `cap` to *unresolved).
cudaError_t launch_fb_gather(const int32_t* ovf, const float* q, const int64_t* probes, int nprobe, int d, int cap,
                             float* fq, int64_t* fprobes, int32_t* fcount, cudaStream_t s);
cudaError_t launch_fb_scatter(const int32_t* ovf, const float* fD, const int64_t* fI, int k, int cap, float* D,
                              int64_t* I, unsigned long long* total, unsigned long long* unresolved, cudaStream_t s);

}  // namespace hy
