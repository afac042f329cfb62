// C-ABI wrapper over the REFERENCE's own C++ code (Harmony's harmony::Index,
// IVFScan, heap and BaseWorker), compiled unmodified from the reference tree
// by oracle/Makefile into oracle/_ref/libharmony_ref.so.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline / reference arm may load this library; the product
// (harmonyclient_b200/libhy.so) never links or calls it.
//
// Entry points (all return 0 on success, -1 on a caught exception, with the
// message available from ref_last_error()):
//   ref_index_new / ref_index_free        harmony::Index ctor (src/Index.h:15-25)
//   ref_train                             Index::train (src/Index.cpp:381-425)
//   ref_set_centroids / ref_get_centroids the public centroid_codes field
//   ref_add                               Index::add (src/Index.cpp:581-697)
//   ref_list_size / ref_get_list          IVF lists (src/IVF.h:17-28)
//   ref_set_opt_level                     the public opt_level field (src/Index.h:108)
//   ref_search_original                   Index::search, ORIGINAL mode
//                                         (src/Index.cpp:1638-1706 -> 1420-1554)
//   ref_probes                            findNearNprobeOfCentroidIds (src/Index.cpp:967-995)
//   ref_warmup_tops                       warmUpSearch + heapTops (src/Index.cpp:999-1051, 1300-1303)
//   ref_search_prune                      BaseWorker::single_thread_search_simple with
//                                         cut=true (src/node.cpp:606-678), heaps initialised
//                                         and sorted as the master does (src/Index.cpp:1309,1340)
//   ref_heap_topk                         heap_replace_top + heap_sort (src/heap.hpp:35-82)
//   ref_search_group                      GROUP mode with pruning, MPI ranks as threads
//                                         (src/Index.cpp:1053-1187, src/node.cpp:679-1203)
//   ref_save / ref_load                   Index::save_index / load_index (src/Index.cpp:1708-1770)
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <memory>
#include <numeric>
#include <queue>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>
#include <omp.h>

// The reference keeps warmUpSearch / findNearNprobeOfCentroidIds private; the
// oracle calls them directly so that the threshold and probe lists can be
// compared one to one with the GPU kernels.
#define private public
#include "Index.h"
#include "heap.hpp"
#include "node.h"
#undef private

using harmony::idx_t;

static thread_local std::string g_err;

extern "C" const char* ref_last_error(void) { return g_err.c_str(); }

#define REF_TRY(body)                    \
    try {                                \
        body;                            \
        return 0;                        \
    } catch (const std::exception& e) {  \
        g_err = e.what();                \
        return -1;                       \
    }

struct RefIndex {
    std::unique_ptr<harmony::Index> idx;
    harmony::Index::Param param;
};

// Discards everything written to it, from any thread (no buffer, so no
// shared put area between threads).
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c == EOF ? 0 : c; }
};

// Silence std::cout while ranks on several threads write to it.
struct QuietAll {
    std::streambuf* old;
    NullBuf sink;
    QuietAll() : old(std::cout.rdbuf(&sink)) {}
    ~QuietAll() { std::cout.rdbuf(old); }
};

// Silence the reference's chatty std::cout while it runs.
struct Quiet {
    std::streambuf* old;
    std::ostringstream sink;
    Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
    ~Quiet() { std::cout.rdbuf(old); }
};

extern "C" int ref_index_new(size_t d, size_t nlist, size_t nprobe, int metric, void** out) {
    REF_TRY({
        auto* r = new RefIndex();
        r->idx = std::make_unique<harmony::Index>(d, nlist, nprobe, static_cast<harmony::MetricType>(metric),
                                                  harmony::OPT_NONE);
        r->idx->added_opt_level = harmony::OPT_NONE;
        r->param.mode = harmony::Index::SearchMode::ORIGINAL;
        r->idx->param = nullptr;
        *out = r;
    });
}

extern "C" void ref_index_free(void* h) { delete static_cast<RefIndex*>(h); }

extern "C" int ref_set_threads(int nt) {
    omp_set_num_threads(nt);
    return 0;
}

extern "C" int ref_train(void* h, size_t n, const float* x, int lite) {
    REF_TRY({
        Quiet q;
        static_cast<RefIndex*>(h)->idx->train(n, x, false, lite != 0);
    });
}

extern "C" int ref_set_centroids(void* h, const float* c) {
    REF_TRY({
        auto& I = *static_cast<RefIndex*>(h)->idx;
        std::copy_n(c, I.nlist * I.d, I.centroid_codes.get());
    });
}

extern "C" int ref_get_centroids(void* h, float* c) {
    REF_TRY({
        auto& I = *static_cast<RefIndex*>(h)->idx;
        std::copy_n(I.centroid_codes.get(), I.nlist * I.d, c);
    });
}

extern "C" int ref_set_nprobe(void* h, size_t nprobe) {
    REF_TRY({ static_cast<RefIndex*>(h)->idx->nprobe = nprobe; });
}

// The public opt_level field (src/Index.h:108): add() stores the per-row
// candidate2centroid for OPT_TRIANGLE (src/Index.cpp:659-667) and the inner
// product search scans the cos-bound window (src/Index.cpp:1509-1546).
extern "C" int ref_set_opt_level(void* h, int opt_level) {
    REF_TRY({ static_cast<RefIndex*>(h)->idx->opt_level = static_cast<harmony::OptLevel>(opt_level); });
}

extern "C" int ref_add(void* h, size_t n, const float* x) {
    REF_TRY({
        Quiet q;
        static_cast<RefIndex*>(h)->idx->add(n, x);
    });
}

extern "C" int ref_list_size(void* h, size_t list, size_t* size) {
    REF_TRY({ *size = static_cast<RefIndex*>(h)->idx->lists[list].get_list_size(); });
}

extern "C" int ref_get_list(void* h, size_t list, int64_t* ids, float* codes, float* norms) {
    REF_TRY({
        auto& I = *static_cast<RefIndex*>(h)->idx;
        auto& L = I.lists[list];
        size_t n = L.get_list_size();
        for (size_t i = 0; i < n; i++) ids[i] = static_cast<int64_t>(L.candidate_id[i]);
        if (codes) std::copy_n(L.candidate_codes.get(), n * I.d, codes);
        if (norms && L.candidate_norms) std::copy_n(L.candidate_norms.get(), n, norms);
    });
}

extern "C" int ref_search_original(void* h, size_t n, const float* q, size_t k, float* D, int64_t* I) {
    REF_TRY({
        Quiet qq;
        auto* r = static_cast<RefIndex*>(h);
        r->param.mode = harmony::Index::SearchMode::ORIGINAL;
        r->param.divideIVFVersionOriginal = false;
        r->idx->preSearch(0, 0, 0, 0, 0, &r->param, "");
        r->idx->search(n, q, k, D, reinterpret_cast<idx_t*>(I));
    });
}

extern "C" int ref_probes(void* h, size_t n, const float* q, int64_t* probes) {
    REF_TRY({
        auto* r = static_cast<RefIndex*>(h);
        auto& I = *r->idx;
        r->param.hardInBalance = false;
        I.param = &r->param;
        if (I.nprobe > I.nlist) I.nprobe = I.nlist;
        I.findNearNprobeOfCentroidIds(n, q);
        std::copy_n(I.listidqueries.get(), n * I.nprobe, probes);
    });
}

// heapTops exactly as the GROUP/IVF masters derive them: run warmUpSearch into
// freshly initialised heaps and read each heap's top (src/Index.cpp:1300-1303).
extern "C" int ref_warmup_tops(void* h, size_t n, const float* q, size_t k, size_t warmup_list,
                               size_t warmup_list_size, const int64_t* probes, float* tops) {
    REF_TRY({
        Quiet qq;
        auto& I = *static_cast<RefIndex*>(h)->idx;
        std::vector<float> D(n * k);
        std::vector<idx_t> L(n * k);
        harmony::init_result(I.metric, n * k, D.data(), L.data());
        I.warmUpSearchList = warmup_list;
        I.warmUpSearchListSize = warmup_list_size;
        std::vector<idx_t> pr(probes, probes + n * I.nprobe);
        I.warmUpSearch(n, q, k, D.data(), L.data(), pr.data());
        for (size_t i = 0; i < n; i++) tops[i] = D[i * k];
    });
}

// The in-rank 4-chunk partial-distance pruning scan (BaseWorker, DIVIDE_IVF)
// run over every list of the index: one "rank" owning lists [0, nlist).
extern "C" int ref_search_prune(void* h, size_t n, const float* q, size_t k, const int64_t* probes,
                                const float* tops, float* D, int64_t* I) {
    REF_TRY({
        auto* r = static_cast<RefIndex*>(h);
        harmony::BaseWorker w;
        w.info = harmony::BaseWorker::InitInfo(r->idx->d, 1, r->idx->nlist, r->idx->nprobe, 0, 0, r->idx->nlist);
        // BaseWorker indexes lists relative to startIVFId through its own Index;
        // lend it ours for the duration of the call.
        w.index.reset(r->idx.release());
        w.cut = true;
        std::vector<idx_t> pr(probes, probes + n * w.info.nprobe);
        std::vector<float> hp(tops, tops + n);
        harmony::init_result(harmony::METRIC_L2, n * k, D, reinterpret_cast<idx_t*>(I));
        w.single_thread_search_simple(n, q, k, D, reinterpret_cast<idx_t*>(I), pr.data(), hp.data());
        for (size_t i = 0; i < n; i++)
            harmony::sort_result(harmony::METRIC_L2, k, D + i * k, reinterpret_cast<idx_t*>(I) + i * k);
        r->idx.reset(w.index.release());
    });
}

// Top-k of a stream of (value, id) pairs through the reference's heap:
// heap_init, heap_replace_top under the caller's strict comparison, heap_sort.
extern "C" int ref_heap_topk(int metric, size_t n, const float* vals, const int64_t* ids, size_t k, float* out_v,
                             int64_t* out_i) {
    REF_TRY({
        harmony::init_result(static_cast<harmony::MetricType>(metric), k, out_v, reinterpret_cast<idx_t*>(out_i));
        for (size_t i = 0; i < n; i++) {
            if (metric == harmony::METRIC_L2) {
                if (vals[i] < out_v[0])
                    harmony::heap_replace_top<harmony::METRIC_L2>(k, out_v, reinterpret_cast<idx_t*>(out_i), vals[i],
                                                                  ids[i]);
            } else {
                if (vals[i] > out_v[0])
                    harmony::heap_replace_top<harmony::METRIC_IP>(k, out_v, reinterpret_cast<idx_t*>(out_i), vals[i],
                                                                  ids[i]);
            }
        }
        harmony::sort_result(static_cast<harmony::MetricType>(metric), k, out_v, reinterpret_cast<idx_t*>(out_i));
    });
}

// The reference's default distributed mode, GROUP with pruning
// (src/Index.cpp:1053-1187 master, src/node.cpp:679-1203 GroupWorker), with
// its MPI ranks as threads of this process (ref_mpi_threads.cpp): rank 0 is
// the calling thread and runs preSearch + search as the benchmark driver's
// master does (src/query.cpp:900-923); ranks 1..workers run what its
// workers run in benchmark mode (src/query.cpp:98-114, 252-255: a barrier,
// then GroupWorker init, receiveQuery, search).  teamSize = workers /
// teamCount as the driver computes it (src/query.cpp:231).  Each worker's
// OpenMP regions use threads_per_rank threads, the master's at least
// team_count.  *seconds receives the wall
// time of the master's Index::search alone (what the reference times).
extern "C" void ref_mpi_threads_init(int size);
extern "C" void ref_mpi_threads_bind(int rank);

extern "C" int ref_search_group(void* h, size_t n, const float* q, size_t k, int workers, int group_count,
                                int team_count, int block_count, size_t warmup_list, size_t warmup_list_size,
                                int cut, int threads_per_rank, const char* scratch_path, float* D, int64_t* I,
                                double* seconds) {
    REF_TRY({
        if (workers < 1 || team_count < 1 || group_count < 1 || block_count < 1 || workers % team_count)
            throw std::runtime_error("ref_search_group: need workers divisible by team_count, all >= 1");
        QuietAll qq;
        auto* r = static_cast<RefIndex*>(h);
        ref_mpi_threads_init(workers + 1);
        std::vector<std::thread> ranks;
        std::vector<std::string> errs(workers + 1);
        for (int rank = 1; rank <= workers; ++rank) {
            ranks.emplace_back([=, &errs] {
                try {
                    ref_mpi_threads_bind(rank);
                    omp_set_num_threads(threads_per_rank);
                    MPI_Barrier(MPI_COMM_WORLD);
                    harmony::GroupWorker w;
                    w.init(rank, false);
                    w.receiveQuery();
                    w.search(cut != 0, false);
                } catch (const std::exception& e) {
                    errs[rank] = e.what();
                }
            });
        }
        ref_mpi_threads_bind(0);
        // The master receives each team's results in an OpenMP loop over the
        // teams and forwards a group's heaps to the next team from inside it
        // (src/Index.cpp:1133-1176): with fewer threads than teams, a team
        // would wait on heaps the master has not reached yet.
        omp_set_num_threads(std::max(threads_per_rank, team_count));
        harmony::Index::Param& p = r->param;
        p.mode = harmony::Index::SearchMode::DIVIDE_GROUP;
        p.orderOptimize = true;
        p.pruning = cut != 0;
        p.fullWarmUp = false;
        p.groupCount = group_count;
        p.teamCount = team_count;
        p.teamSize = workers / team_count;
        p.hardInBalance = false;
        size_t nb = 0;
        for (size_t l = 0; l < r->idx->nlist; ++l) nb += r->idx->lists[l].get_list_size();
        try {
            // The driver's barrier before preSearch (src/query.cpp:900) meets
            // the workers' first one; preSearch's own closing barrier meets
            // the one that opens GroupWorker::receiveQuery (src/node.cpp:766).
            if (MPI_Barrier(MPI_COMM_WORLD) != 0) throw std::runtime_error("GROUP: barrier before preSearch");
            r->idx->preSearch(nb, workers, block_count, warmup_list, warmup_list_size, &p, scratch_path);
            const auto t0 = std::chrono::steady_clock::now();
            r->idx->search(n, q, k, D, reinterpret_cast<idx_t*>(I));
            *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        } catch (...) {
            for (auto& t : ranks) t.join();
            ref_mpi_threads_init(1);
            throw;
        }
        for (auto& t : ranks) t.join();
        ref_mpi_threads_init(1);
        omp_set_num_threads(omp_get_num_procs());
        for (const auto& e : errs)
            if (!e.empty()) throw std::runtime_error("GROUP worker: " + e);
    });
}

extern "C" int ref_save(void* h, const char* path) {
    REF_TRY({ static_cast<RefIndex*>(h)->idx->save_index(path); });
}

extern "C" int ref_load(void* h, const char* path) {
    REF_TRY({
        Quiet q;
        static_cast<RefIndex*>(h)->idx->load_index(path);
    });
}

extern "C" int ref_info(void* h, size_t* d, size_t* nlist, size_t* nprobe, int* metric) {
    REF_TRY({
        auto& I = *static_cast<RefIndex*>(h)->idx;
        *d = I.d;
        *nlist = I.nlist;
        *nprobe = I.nprobe;
        *metric = static_cast<int>(I.metric);
    });
}

// ---------------------------------------------------------------------------
// The reference's dataset / result-file readers and recall metrics
// (src/utils.h:187-407, 565-756), for the golden fixtures of
// harmonyclient_b200/datafiles.py.
static void xvecs_info(const char* path, size_t* n, int* d) {
    const std::pair<size_t, int> r = harmony::loadXvecsInfo(path);
    *n = r.first;
    *d = r.second;
}

extern "C" int ref_xvecs_info(const char* path, size_t* n, int* d) { REF_TRY({ xvecs_info(path, n, d); }); }

static void load_xvecs(const char* path, int a, int b, float* out, size_t cap, size_t* n, int* d) {
    auto t = harmony::loadXvecs(path, std::make_pair(a, b));
    const size_t nn = std::get<1>(t);
    const int dd = std::get<2>(t);
    if (nn * static_cast<size_t>(dd) > cap) throw std::runtime_error("ref_load_xvecs: output too small");
    std::memcpy(out, std::get<0>(t).get(), nn * static_cast<size_t>(dd) * sizeof(float));
    *n = nn;
    *d = dd;
}

// Rows a..b (1-based, b = 0: to the end) of a .fvecs / .bvecs / .txt file as
// float32 (the reference's loadXvecs); out must hold cap floats.
extern "C" int ref_load_xvecs(const char* path, int a, int b, float* out, size_t cap, size_t* n, int* d) {
    REF_TRY({ load_xvecs(path, a, b, out, cap, n, d); });
}

extern "C" int ref_write_results(const int64_t* labels, const float* distances, size_t nq, size_t k,
                                 const char* path) {
    REF_TRY({ harmony::writeResultsToFile(reinterpret_cast<const idx_t*>(labels), distances, nq, k, path); });
}

extern "C" int ref_load_results(const char* path, int64_t* labels, float* distances, size_t nq, size_t k) {
    REF_TRY({ harmony::loadResults(path, reinterpret_cast<idx_t*>(labels), distances, nq, k); });
}

// which: 0 calculate_recall, 1 calculate_recall_loose, 2 calculate_r2.
static float recall_of(int which, const int64_t* I, const float* D, const int64_t* GT, const float* GD, size_t nq,
                       size_t k, int metric, size_t gt_k) {
    const auto m = static_cast<harmony::MetricType>(metric);
    const auto* i = reinterpret_cast<const idx_t*>(I);
    const auto* g = reinterpret_cast<const idx_t*>(GT);
    Quiet q;
    if (which == 0) return harmony::calculate_recall(i, D, g, GD, nq, k, m, gt_k);
    if (which == 1) return harmony::calculate_recall_loose(i, D, g, GD, nq, k, m, gt_k);
    return harmony::calculate_r2(i, D, g, GD, nq, k, m, gt_k);
}

extern "C" int ref_recall(int which, const int64_t* I, const float* D, const int64_t* GT, const float* GD, size_t nq,
                          size_t k, int metric, size_t gt_k, float* out) {
    REF_TRY({ *out = recall_of(which, I, D, GT, GD, nq, k, metric, gt_k); });
}
