// harmony::Index over the B200 engine — a header-only C++ facade with the
// reference's class interface (src/Index.h:11-149 of the Harmony repository),
// so code written against Harmony's Index compiles against this header and
// links against libhy.so instead.
//
// Kept from the reference: the constructor's argument list and defaults
// (src/Index.h:15-25), default construction and move assignment (the
// benchmark driver's `Index index; index = Index(...)`, src/query.cpp:830-837),
// train / add / search / preSearch / postSearch / save_index / load_index
// (src/Index.h:69-91), Param, SearchMode and to_string (src/Index.h:29-68),
// the public fields callers read and write: nprobe / nlist / d, centroid_codes
// as std::unique_ptr<float[]> (src/Index.h:118, read through .get() by
// src/node.cpp:50), lists as per-list IVF objects with the reference's
// accessors (src/IVF.h:9-75, read by src/query.cpp:617-618), trainTime /
// addTime / preSearchTime in seconds (src/Index.h:148, read by
// src/query.cpp:768-770); MetricType / OptLevel / EdgeDevice
// (src/common.h:20-32); Stats as search's return type with the reference's
// public fields, print() and myToCsv() (src/stats.h:14-134).  Errors throw
// std::runtime_error, as the reference does (src/Index.cpp:60, 1644).
//
// Differences, by design: everything runs on one GPU through the C-ABI;
// centroid_codes is synchronised with the device when add / search /
// save_index run (write it, then call add or search, as callers of the
// reference do); lists are read back from the device the first time a list
// is indexed after add / load_index; preSearch's worker / block counts
// describe MPI partitions that do not exist on one GPU, so only its warm-up
// parameters are used; Stats' triangle / sub-NN counters stay 0 (those opt
// levels are not counted) and its engine counters are extra fields; the
// number of dimension blocks used for pruning is a constructor extra
// (default 4, the reference's fixed value, src/node.cpp:639).
#ifndef HARMONY_B200_INDEX_H
#define HARMONY_B200_INDEX_H

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
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

inline void hy_throw_if(int rc) {
    if (rc != HY_OK) throw std::runtime_error(std::string("hy: ") + hy_last_error());
}

// Search statistics.  The reference's public fields (src/stats.h:14-50) are
// here for callers that fill and print them; search() sets nq, nlist, nprobe,
// d, k, query_time and the engine's counters.
class Stats {
   public:
    size_t total_count = 0;
    size_t skip_triangle_count = 0, skip_triangle_large_count = 0;
    size_t check_subnn_L2_ele_count = 0, check_subnn_IP_ele_count = 0;
    size_t check_subnn_L2_count = 0, check_subnn_IP_count = 0;
    size_t skip_subnn_L2_count = 0, skip_subnn_IP_count = 0;
    size_t simi_update_count = 0, dis_calculate_count = 0;
    size_t nlist = 0;
    size_t nq = 0, nb = 0, d = 0, k = 0;
    size_t nprobe = 0;
    std::string mode = "Original";
    bool divideIVF = false, disableOrderOptimize = false, pruning = false, blockSend = false;
    size_t block = 0, worker = 0, group = 0, team = 0;
    double blockVersionSpeedUpWithOriginal = 0;
    double faiss_query_time = 0;
    double query_time = 0, original_time = 0;
    double trainTime = 0, addTime = 0, preSearchTime = 0, inBalanceRatio = 0, inBalanceRatioTeam = 0;
    double brute_ratio = 0;
    OptLevel opt_level = OPT_NONE;
    double recall = 0, recall_loose = 0;
    double r2 = 0;
    double variance = 0;
    float simi_ratio = 0;

    // Engine counters (no counterpart in the reference).
    uint64_t pairs = 0;                             // (query, probed list) pairs
    uint64_t tile_blocks = 0, tile_blocks_max = 0;  // dimension blocks loaded / without pruning
    double coarse_ms = 0, scan_ms = 0, merge_ms = 0;
    uint64_t fallback_queries = 0;
    double skip_rate() const {
        return tile_blocks_max ? 1.0 - double(tile_blocks) / double(tile_blocks_max) : 0.0;
    }

    double time_speedup() const { return query_time == 0 ? 0 : 100.0 * faiss_query_time / query_time; }

    void print() const {
        std::cout << "nprobe:" << nprobe << " opt_level: " << static_cast<int>(opt_level)
                  << " simi_ratio: " << simi_ratio << "\n"
                  << "time_speedup: " << fixed(time_speedup(), 2) << "% faiss_query_time: "
                  << fixed(faiss_query_time, 6) << " query_time: " << fixed(query_time, 6) << "\n"
                  << "recall: " << recall << " r2: " << r2 << "\n";
    }

    // One row of the reference's benchmark log (src/stats.h:122-134): the
    // header first unless appending to an existing file; floats with 7
    // decimals, doubles with 16, booleans as 1 / 0 (src/utils.h:41-140).
    void myToCsv(const std::string& filename, bool append, const std::string& dataset = "Unknown") const {
        static const char* cols[] = {"dataset", "mode", "nb", "nq", "d", "nlist", "nprobe", "k", "divideIVF",
                                     "orderOptimize", "UnblockSend", "cut", "block", "worker", "group", "team",
                                     "time_speedup", "query_time", "original_time", "recall", "r2", "variance",
                                     "train_time", "add_time", "preSearch_time", "ratio", "teamRatio", "brute_ratio"};
        const bool exists = std::ifstream(filename).good();
        std::ofstream f(filename, append && exists ? std::ios::app : std::ios::trunc);
        if (!f) throw std::runtime_error("hy: cannot write " + filename);
        if (!(append && exists)) {
            for (size_t i = 0; i < sizeof(cols) / sizeof(cols[0]); ++i) f << (i ? "," : "") << cols[i];
            f << "\n";
        }
        f << dataset << "," << mode << "," << nb << "," << nq << "," << d << "," << nlist << "," << nprobe << ","
          << k << "," << int(divideIVF) << "," << int(!disableOrderOptimize) << "," << int(!blockSend) << ","
          << int(pruning) << "," << block << "," << worker << "," << group << "," << team << ","
          << fixed(time_speedup(), 16) << "," << fixed(query_time, 16) << "," << fixed(original_time, 16) << ","
          << fixed(recall, 16) << "," << fixed(r2, 16) << "," << fixed(variance, 16) << "," << fixed(trainTime, 16)
          << "," << fixed(addTime, 16) << "," << fixed(preSearchTime, 16) << "," << fixed(inBalanceRatio, 16) << ","
          << fixed(inBalanceRatioTeam, 16) << "," << fixed(brute_ratio, 16) << "\n";
    }

   private:
    static std::string fixed(double v, int digits) {
        std::ostringstream o;
        o.setf(std::ios::fixed);
        o.precision(digits);
        o << v;
        return o.str();
    }
};

// One inverted list as the reference's IVF exposes it (src/IVF.h:9-75):
// ids (candidate_id, the row index passed to add), row-major codes and
// squared norms, read back from the device.
class IVF {
   public:
    size_t list_size = 0;
    size_t d = 0;
    size_t sub_k = 0;
    OptLevel opt_level = OPT_NONE;
    std::unique_ptr<size_t[]> candidate_id;
    std::unique_ptr<float[]> candidate_codes;
    std::unique_ptr<float[]> candidate_norms;

    size_t get_list_size() const { return list_size; }
    size_t get_d() const { return d; }
    size_t get_sub_k() const { return sub_k; }
    const float* get_candidate_codes() const { return candidate_codes.get(); }
    const float* get_candidate_codes(size_t i) const { return candidate_codes.get() + i * d; }
    const size_t* get_candidate_id() const { return candidate_id.get(); }
    size_t get_candidate_id(size_t i) const { return candidate_id[i]; }
    const float* get_candidate_norms() const { return candidate_norms.get(); }
};

// index.lists[l]: list l, read from the device on first use after each
// add / load_index.
class ListTable {
   public:
    IVF& operator[](size_t l) {
        if (!h_) throw std::runtime_error("hy: index has no lists");
        if (l >= loaded_.size()) {
            hy_index_info_t inf{};
            hy_throw_if(hy_index_info(h_, &inf));
            if (l >= inf.nlist) throw std::out_of_range("hy: list id out of range");
            lists_.reset(new IVF[inf.nlist]);
            loaded_.assign(inf.nlist, 0);
            d_ = inf.d;
        }
        IVF& v = lists_[l];
        if (!loaded_[l]) {
            size_t n = 0;
            hy_throw_if(hy_index_list_size(h_, l, &n));
            std::vector<int64_t> ids(n);
            v.list_size = n;
            v.d = d_;
            v.candidate_id.reset(new size_t[n]);
            v.candidate_codes.reset(new float[n * d_]);
            v.candidate_norms.reset(new float[n]);
            if (n) hy_throw_if(hy_index_get_list(h_, l, ids.data(), v.candidate_codes.get(), v.candidate_norms.get()));
            for (size_t i = 0; i < n; ++i) v.candidate_id[i] = static_cast<size_t>(ids[i]);
            loaded_[l] = 1;
        }
        return v;
    }
    void reset(hy_index* h) {
        h_ = h;
        lists_.reset();
        loaded_.clear();
    }

   private:
    hy_index* h_ = nullptr;
    size_t d_ = 0;
    std::unique_ptr<IVF[]> lists_;
    std::vector<char> loaded_;
};

class Index {
   public:
    enum class SearchMode { BRUTE_FORCE, ORIGINAL, DIVIDE_IVF, DIVIDE_DIM, DIVIDE_GROUP };

    static std::string to_string(SearchMode mode) {
        switch (mode) {
            case SearchMode::BRUTE_FORCE: return "Brute Force";
            case SearchMode::ORIGINAL: return "Original";
            case SearchMode::DIVIDE_IVF: return "Baseline";
            case SearchMode::DIVIDE_DIM: return "Dim     ";
            case SearchMode::DIVIDE_GROUP: return "Group   ";
        }
        return "Unknown";
    }

    // The reference's search parameters (src/Index.h:48-68).  The partition
    // fields describe its MPI modes; on one GPU the search is the same exact
    // scan with dimension-block pruning whatever they hold.
    struct Param {
        bool orderOptimize = true;
        SearchMode mode = SearchMode::ORIGINAL;
        bool divideIVFVersionOriginal = false;
        size_t startIVFId = 0, ivfCount = 0;
        size_t block_dim = 0;
        idx_t* queryCompareSize = nullptr;
        idx_t* queryCompareSizePreSum = nullptr;
        idx_t queryStart = 0;
        idx_t* listidqueries = nullptr;
        bool pruning = false;
        bool period = false;
        bool fullWarmUp = false;
        float* heapTops = nullptr;
        size_t groupCount = 1, teamCount = 1, teamSize = 1;
        bool hardInBalance = false;
        size_t hardInBalanceTeam = 0;
        float hardInBalanceRatio = 0;
        float hardInBalanceTeamRatio = 0;
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
    Index(Index&& o) noexcept { *this = std::move(o); }
    Index& operator=(Index&& o) noexcept {
        if (this != &o) {
            hy_index_destroy(h_);
            h_ = o.h_;
            o.h_ = nullptr;
            d = o.d;
            nlist = o.nlist;
            nprobe = o.nprobe;
            workerCount = o.workerCount;
            blockCount = o.blockCount;
            metric = o.metric;
            opt_level = o.opt_level;
            sub_k = o.sub_k;
            sub_nlist = o.sub_nlist;
            sub_nprobe = o.sub_nprobe;
            verbose = o.verbose;
            edge_device_enabled = o.edge_device_enabled;
            centroid_codes = std::move(o.centroid_codes);
            trainTime = o.trainTime;
            addTime = o.addTime;
            preSearchTime = o.preSearchTime;
            dim_blocks_ = o.dim_blocks_;
            device_ = o.device_;
            param_ = o.param_;
            synced_ = std::move(o.synced_);
            lists.reset(h_);
            o.lists.reset(nullptr);
        }
        return *this;
    }

    // src/Index.cpp:381-425.  `faiss` training is not part of this engine.
    void train(size_t n, const float* codes, bool faiss = false, bool lite = false) {
        if (faiss) throw std::runtime_error("hy: faiss training is not available");
        const auto t0 = std::chrono::steady_clock::now();
        hy_throw_if(hy_index_train(h_, n, codes, lite ? 1 : 0));
        pull_centroids();
        trainTime = seconds_since(t0);
    }

    // src/Index.cpp:581-697: rebuilds the lists from these rows (ids 0..n-1).
    void add(size_t n, const float* codes) {
        const auto t0 = std::chrono::steady_clock::now();
        push_centroids();
        hy_throw_if(hy_index_add(h_, n, codes));
        lists.reset(h_);
        addTime = seconds_since(t0);
    }

    // src/Index.h:90: only the warm-up parameters apply on one GPU.
    void preSearch(size_t /*nb*/, size_t workerCount_, size_t blockCount_, size_t warmUpSearchList,
                   size_t warmUpSearchListSize, Param* param, std::string /*path*/) {
        const auto t0 = std::chrono::steady_clock::now();
        workerCount = workerCount_;
        blockCount = blockCount_;
        param_ = param;
        hy_throw_if(hy_index_presearch(h_, warmUpSearchList, warmUpSearchListSize));
        preSearchTime = seconds_since(t0);
    }
    void postSearch() {}

    // src/Index.cpp:1638-1706.  distances / labels are n x k, best first.
    Stats search(size_t n, const float* queries, size_t k, float* distances, idx_t* labels, float /*ratio*/ = 1) {
        const auto t0 = std::chrono::steady_clock::now();
        push_centroids();
        hy_throw_if(hy_index_set_nprobe(h_, nprobe ? nprobe : 1));
        hy_throw_if(hy_index_set_opt_level(h_, static_cast<int>(opt_level)));
        hy_throw_if(hy_index_search(h_, n, queries, k, distances, labels));
        hy_search_stats_t st{};
        hy_throw_if(hy_index_last_stats(h_, &st));
        Stats s;
        s.nq = st.nq;
        s.nlist = nlist;
        s.nprobe = nprobe;
        s.d = d;
        s.k = k;
        s.opt_level = opt_level;
        s.mode = to_string(param_ ? param_->mode : SearchMode::ORIGINAL);
        s.pruning = param_ ? param_->pruning : false;
        s.trainTime = trainTime;
        s.addTime = addTime;
        s.preSearchTime = preSearchTime;
        s.pairs = st.pairs;
        s.tile_blocks = st.tile_blocks;
        s.tile_blocks_max = st.tile_blocks_max;
        s.coarse_ms = st.coarse_ms;
        s.scan_ms = st.scan_ms;
        s.merge_ms = st.merge_ms;
        s.fallback_queries = st.fallback_queries;
        s.total_count = static_cast<size_t>(st.rows);
        s.query_time = seconds_since(t0);
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
        if (!h_) {
            // A default-constructed Index (src/query.cpp:830-833) learns its
            // shape from the file.
            size_t fd = 0, fnl = 0, nonempty = 0, total = 0;
            int fm = 0, fopt = 0;
            hy_throw_if(hy_file_inspect(path.c_str(), &fd, &fnl, &fm, &fopt, &nonempty, &total));
            d = fd;
            nlist = fnl;
            metric = static_cast<MetricType>(fm);
            create();
        }
        hy_throw_if(hy_index_load(h_, path.c_str()));
        hy_index_info_t inf{};
        hy_throw_if(hy_index_info(h_, &inf));
        d = inf.d;
        nlist = inf.nlist;
        metric = static_cast<MetricType>(inf.metric);
        opt_level = OPT_NONE;
        pull_centroids();
        lists.reset(h_);
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

    size_t d = 0;
    size_t nlist = 0;
    size_t nprobe = 0;
    size_t workerCount = 0;
    size_t blockCount = 0;
    MetricType metric = METRIC_L2;
    OptLevel opt_level = OPT_NONE;
    size_t sub_k = 0, sub_nlist = 1, sub_nprobe = 1;
    bool verbose = false;
    EdgeDevice edge_device_enabled = EDGEDEVIVE_DISABLED;
    ListTable lists;                          // lists[l] (src/Index.h:117)
    std::unique_ptr<float[]> centroid_codes;  // nlist x d, row-major (src/Index.h:118)
    double trainTime = 0, addTime = 0, preSearchTime = 0;

   private:
    static double seconds_since(std::chrono::steady_clock::time_point t0) {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void create() {
        hy_throw_if(hy_index_create(d, nlist, nprobe, static_cast<int>(metric), static_cast<int>(opt_level),
                                    dim_blocks_, device_, &h_));
        centroid_codes.reset(new float[nlist * d]());
        synced_.assign(nlist * d, 0.0f);
        lists.reset(h_);
    }
    void pull_centroids() {
        if (!centroid_codes || synced_.size() != nlist * d) centroid_codes.reset(new float[nlist * d]);
        synced_.resize(nlist * d);
        hy_throw_if(hy_index_get_centroids(h_, centroid_codes.get()));
        std::memcpy(synced_.data(), centroid_codes.get(), synced_.size() * sizeof(float));
    }
    // Callers of the reference write centroid_codes directly (through .get()
    // or a new array); hand any change to the engine before it is used.
    void push_centroids() {
        if (!centroid_codes || synced_.size() != nlist * d) return;
        if (std::memcmp(synced_.data(), centroid_codes.get(), synced_.size() * sizeof(float)) != 0) {
            hy_throw_if(hy_index_set_centroids(h_, centroid_codes.get()));
            std::memcpy(synced_.data(), centroid_codes.get(), synced_.size() * sizeof(float));
        }
    }

    hy_index* h_ = nullptr;
    size_t dim_blocks_ = 4;
    int device_ = 0;
    Param* param_ = nullptr;
    std::vector<float> synced_;
};

}  // namespace harmony

#endif  // HARMONY_B200_INDEX_H
