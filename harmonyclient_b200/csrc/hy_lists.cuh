// Host-visible launchers of the list-major exact FP32 scan (hy_lists.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hy_kernels.cuh"

namespace hy {

// Queries per group of the list-major scan (one bit per query in a lane's
// live mask).
constexpr int LM_GROUP = 32;

struct ListScanParams {
    ArenaLayout L;
    const float* codes;         // FP32 arena
    const int64_t* list_off;    // [nlist+1] first arena row of each list
    const int32_t* list_size;   // [nlist]
    const float* q;             // [nq][d]
    const int64_t* item_off;    // [nlist+1] first work item of each list
    const int4* items;          // [item_cap] {list, query group, row slice}
    int64_t item_cap;
    const int64_t* pair_off;    // [nlist+1]
    const int32_t* pairs;       // query ids grouped by list
    const int32_t* pair_cnt;    // [nlist]
    const uint32_t* thr;        // [nq] ordered-key thresholds (0xffffffff: none), or nullptr
    uint64_t* cand;             // [nq][capq] candidate keys (ordered score << 32 | arena row)
    int32_t* cand_cnt;          // [nq]
    unsigned int* work;         // work-queue counter (zero before the launch)
    // [4]: block copies, block copies without pruning, executed (query,
    // 32-row tile, 16-dimension segment) partial sums, and those without pruning
    unsigned long long* counters;
    int* err;
    int nlist, rs, capq, metric, prune;
    int qg = LM_GROUP;          // queries per group the items were built with
    // Centroid windows: per arena row its L2 distance to (L2) or inner
    // product with (inner product, OPT_TRIANGLE) its list's centroid, per
    // 32-row tile {max, min} of those, the centroids.
    int triangle = 0;
    const float* c2c = nullptr;
    const float2* c2c_tile = nullptr;
    const float* cent = nullptr;
};

// True when some dimension block is wider than 32 floats (the multi-chunk
// kernel variant).
bool list_scan_multi(const ArenaLayout& L);
// True when the scan's shared memory (block-copy slots and the group's
// queries) fits one CTA for this layout.
bool list_scan_fits(const ArenaLayout& L);
// Persistent launch (nsm x the CTAs per SM that fit).
cudaError_t launch_list_scan(const ListScanParams& p, int nsm, cudaStream_t s);
// c2c [arena rows] := each valid row's L2 distance to (metric L2, not
// squared) or inner product with (inner product) its list's centroid;
// c2c_tile [arena rows / 32] := {max, min} over each tile's valid rows
// (lists start on 32-row tiles).
cudaError_t launch_row_centroid(const ArenaLayout& L, const float* codes, const int64_t* list_off,
                                const int32_t* list_size, int nlist, int64_t arena_rows, const float* cent, int metric,
                                float* c2c, float2* c2c_tile, cudaStream_t s);
// mode 0: keep each query's k best candidates and lower its threshold to the
// k-th; mode 1: write the k best as (distance, id) into D / I, listing the
// queries whose candidates overflowed in ovf (count first) instead.
cudaError_t launch_list_topk(uint64_t* cand, int32_t* cnt, int nq, int capq, int k, int metric, int mode,
                             uint32_t* thr, const int64_t* ids, float* D, int64_t* I, int32_t* ovf, cudaStream_t s);

}  // namespace hy
