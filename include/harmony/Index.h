// harmony::Index over the B200 engine — a header-only C++ facade with the
// reference's class interface (src/Index.h:11-149 of the Harmony repository),
// so code written against Harmony's Index compiles against this header and
// links against libhy.so instead.
//
// Kept from the reference: the constructor's argument list and defaults
// (src/Index.h:15-25), train / add / search / preSearch / postSearch /
// save_index / load_index (src/Index.h:69-91), the public centroid_codes /
// nprobe / nlist / d fields callers read and write (src/Index.h:99-118,
// src/query.cpp:469-470, 768-770), MetricType / OptLevel / EdgeDevice
// (src/common.h:20-32) and Stats as search's return type.  Errors throw
// std::runtime_error, as the reference does (src/Index.cpp:60, 1644).
//
// Differences, by design: everything runs on one GPU through the C-ABI;
// centroid_codes is synchronised with the device when train/add/search run
// (write it, then call add or search, as callers of the reference do);
// preSearch's worker/block counts describe MPI partitions that do not exist
// on one GPU and only its warm-up parameters are used; the number of
// dimension blocks used for pruning is a constructor extra (default 4, the
// reference's fixed value, src/node.cpp:639).
#ifndef HARMONY_B200_INDEX_H
#define HARMONY_B200_INDEX_H

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../hy.h"

namespace harmony {

enum MetricType { METRIC_IP = 0, METRIC_L2 };

enum OptLevel {
    OPT_NONE = 0b000,
    OPT_TRIANGLE = 0b001,
    OPT_SUBNN_L2 = 0b010,
    OPT_SUBNN_IP = 0b100,
    OPT_TRI_SUBNN_L2 = 0b011,
    OPT_TRI_SUBNN_IP = 0b101,
    OPT_SUBNN_ONLY = 0b110,
    OPT_ALL = 0b111
};

enum EdgeDevice { EDGEDEVIVE_ENABLED, EDGEDEVIVE_DISABLED };

using idx_t = int64_t;

// Counters returned by search (the reference's Stats, src/stats.h, holds
// pruning counters; these are the engine's equivalents).
struct Stats {
    uint64_t nq = 0, pairs = 0;
    uint64_t tile_blocks = 0, tile_blocks_max = 0;  // dimension blocks loaded / possible
    double coarse_ms = 0, scan_ms = 0, merge_ms = 0;
    uint64_t fallback_queries = 0;
    double skip_rate() const {
        return tile_blocks_max ? 1.0 - double(tile_blocks) / double(tile_blocks_max) : 0.0;
    }
};

inline void hy_throw_if(int rc) {
    if (rc != HY_OK) throw std::runtime_error(std::string("hy: ") + hy_last_error());
}

class Index {
   public:
    enum class SearchMode { BRUTE_FORCE, ORIGINAL, DIVIDE_IVF, DIVIDE_DIM, DIVIDE_GROUP };

    struct Param {
        bool orderOptimize = true;
        SearchMode mode = SearchMode::ORIGINAL;
        bool pruning = false;
        size_t groupCount = 1, teamCount = 1, teamSize = 1;
    };

    Index(size_t d = 0, size_t nlist = 0, size_t nprobe = 0, MetricType metric = METRIC_L2,
          OptLevel opt_level = OPT_NONE, size_t sub_k = 0, size_t sub_nlist = 1, size_t sub_nprobe = 1,
          bool verbose = false, EdgeDevice edge_device_enabled = EDGEDEVIVE_DISABLED, size_t dim_blocks = 4,
          int device = 0)
        : d(d),
          nlist(nlist),
          nprobe(nprobe),
          metric(metric),
          opt_level(opt_level),
          sub_k(sub_k),
          sub_nlist(sub_nlist),
          sub_nprobe(sub_nprobe),
          verbose(verbose),
          edge_device_enabled(edge_device_enabled),
          dim_blocks_(dim_blocks),
          device_(device) {
        if (d && nlist) create();
    }

    ~Index() { hy_index_destroy(h_); }
    Index(const Index&) = delete;
    Index& operator=(const Index&) = delete;
    Index& operator=(Index&& o) noexcept {
        if (this != &o) {
            hy_index_destroy(h_);
            h_ = o.h_;
            o.h_ = nullptr;
            d = o.d;
            nlist = o.nlist;
            nprobe = o.nprobe;
            metric = o.metric;
            opt_level = o.opt_level;
            centroid_codes = std::move(o.centroid_codes);
            synced_ = std::move(o.synced_);
        }
        return *this;
    }

    // src/Index.cpp:381-425.  `faiss` training is not part of this engine.
    void train(size_t n, const float* codes, bool faiss = false, bool lite = false) {
        if (faiss) throw std::runtime_error("hy: faiss training is not available");
        hy_throw_if(hy_index_train(h_, n, codes, lite ? 1 : 0));
        pull_centroids();
    }

    // src/Index.cpp:581-697: rebuilds the lists from these rows (ids 0..n-1).
    void add(size_t n, const float* codes) {
        push_centroids();
        hy_throw_if(hy_index_add(h_, n, codes));
    }

    // src/Index.h:90: only the warm-up parameters apply on one GPU.
    void preSearch(size_t /*nb*/, size_t /*workerCount*/, size_t /*blockCount*/, size_t warmUpSearchList,
                   size_t warmUpSearchListSize, Param* param, std::string /*path*/) {
        param_ = param;
        hy_throw_if(hy_index_presearch(h_, warmUpSearchList, warmUpSearchListSize));
    }
    void postSearch() {}

    // src/Index.cpp:1638-1706.  distances / labels are n x k, best first.
    Stats search(size_t n, const float* queries, size_t k, float* distances, idx_t* labels, float /*ratio*/ = 1) {
        push_centroids();
        hy_throw_if(hy_index_set_nprobe(h_, nprobe ? nprobe : 1));
        hy_throw_if(hy_index_search(h_, n, queries, k, distances, labels));
        hy_search_stats_t st{};
        hy_throw_if(hy_index_last_stats(h_, &st));
        Stats s;
        s.nq = st.nq;
        s.pairs = st.pairs;
        s.tile_blocks = st.tile_blocks;
        s.tile_blocks_max = st.tile_blocks_max;
        s.coarse_ms = st.coarse_ms;
        s.scan_ms = st.scan_ms;
        s.merge_ms = st.merge_ms;
        s.fallback_queries = st.fallback_queries;
        return s;
    }

    // Scan form: HY_FORM_PLAIN (exact FP32 scan) or HY_FORM_BF16 (batched
    // tensor-core scan with exact FP32 re-rank).  Not in the reference.
    void set_form(int form) { hy_throw_if(hy_index_set_form(h_, form)); }
    // Coarse step of the bf16 form: HY_COARSE_TENSOR (default) or
    // HY_COARSE_EXACT; the probe lists are the same.  Not in the reference.
    void set_coarse(int mode) { hy_throw_if(hy_index_set_coarse(h_, mode)); }
    // Replay repeated searches of one shape as a captured CUDA graph.  Not in
    // the reference.
    void set_graph(bool on) { hy_throw_if(hy_index_set_graph(h_, on ? 1 : 0)); }

    void save_index(std::string path) const {
        const_cast<Index*>(this)->push_centroids();
        hy_throw_if(hy_index_save(h_, path.c_str()));
    }
    void load_index(std::string path) {
        hy_throw_if(hy_index_load(h_, path.c_str()));
        hy_index_info_t inf{};
        hy_throw_if(hy_index_info(h_, &inf));
        d = inf.d;
        nlist = inf.nlist;
        metric = static_cast<MetricType>(inf.metric);
        opt_level = OPT_NONE;
        pull_centroids();
    }

    size_t list_size(size_t list) const {
        size_t s = 0;
        hy_throw_if(hy_index_list_size(h_, list, &s));
        return s;
    }
    void get_list(size_t list, idx_t* ids, float* codes) const {
        hy_throw_if(hy_index_get_list(h_, list, ids, codes, nullptr));
    }

    hy_index* handle() const { return h_; }

    size_t d;
    size_t nlist;
    size_t nprobe;
    MetricType metric;
    OptLevel opt_level;
    size_t sub_k, sub_nlist, sub_nprobe;
    bool verbose;
    EdgeDevice edge_device_enabled;
    std::vector<float> centroid_codes;  // nlist x d, row-major (src/Index.h:118)
    double trainTime = 0, addTime = 0, preSearchTime = 0;

   private:
    void create() {
        hy_throw_if(hy_index_create(d, nlist, nprobe, static_cast<int>(metric), static_cast<int>(opt_level),
                                    dim_blocks_, device_, &h_));
        centroid_codes.assign(nlist * d, 0.0f);
    }
    void pull_centroids() {
        centroid_codes.resize(nlist * d);
        hy_throw_if(hy_index_get_centroids(h_, centroid_codes.data()));
        synced_ = centroid_codes;
    }
    // Callers of the reference write centroid_codes directly; hand any change
    // to the engine before it is used.
    void push_centroids() {
        if (centroid_codes.size() == nlist * d && centroid_codes != synced_) {
            hy_throw_if(hy_index_set_centroids(h_, centroid_codes.data()));
            synced_ = centroid_codes;
        }
    }

    hy_index* h_ = nullptr;
    size_t dim_blocks_;
    int device_;
    Param* param_ = nullptr;
    std::vector<float> synced_;
};

}  // namespace harmony

#endif  // HARMONY_B200_INDEX_H
