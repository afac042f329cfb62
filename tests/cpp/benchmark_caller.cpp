// A caller written the way the reference's benchmark and serving drivers use
// harmony::Index (src/query.cpp:446-656 and 827-944, src/node.cpp:50,494),
// compiled against include/harmony/Index.h:
//   * `Index index;` then `index = Index(d, nlist, 0, metric, opt, OPT_ALL, ...)`,
//     train, add, save_index; a second default-constructed Index load_index()es
//     the file (the benchmark's --cache path);
//   * the centroids broadcast into `centroid_codes.get()` of a third index
//     (what each MPI worker receives) before its add;
//   * `index.lists[0].get_list_size()` / `.candidate_id[i]` (the serving
//     driver's sample print);
//   * a loop over nprobes: `index.nprobe = np`, Param with the reference's
//     fields, preSearch, search, Stats fields filled and myToCsv;
//   * trainTime / addTime / preSearchTime.
// Writes what it saw for the test to check:
//   benchmark_caller <d> <nlist> <k> <base.f32> <nb> <queries.f32> <nq> <dir>
// <dir>/I_<np>_{a,b,c}.i64 and D_<np>_{a,b,c}.f32 for nprobe np in {1, 4, nlist},
// <dir>/list0.i64, <dir>/C.f32 (centroids), <dir>/log.csv, <dir>/times.txt.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <vector>

#include "harmony/Index.h"

using namespace harmony;

template <class T>
static std::unique_ptr<T[]> read_raw(const std::string& path, size_t n) {
    std::unique_ptr<T[]> v(new T[n]);
    std::ifstream in(path, std::ios::binary);
    in.read(reinterpret_cast<char*>(v.get()), static_cast<std::streamsize>(n * sizeof(T)));
    if (!in) throw std::runtime_error("cannot read " + path);
    return v;
}

template <class T>
static void write_raw(const std::string& path, const T* p, size_t n) {
    std::ofstream(path, std::ios::binary).write(reinterpret_cast<const char*>(p), n * sizeof(T));
}

int main(int argc, char** argv) {
    if (argc < 9) {
        std::fprintf(stderr, "usage: benchmark_caller d nlist k base nb queries nq dir\n");
        return 2;
    }
    const size_t d = std::strtoul(argv[1], nullptr, 10), nlist = std::strtoul(argv[2], nullptr, 10);
    const size_t k = std::strtoul(argv[3], nullptr, 10);
    const size_t nb = std::strtoul(argv[5], nullptr, 10), nq = std::strtoul(argv[7], nullptr, 10);
    const std::string dir = argv[8];
    try {
        auto base = read_raw<float>(argv[4], nb * d);
        auto query = read_raw<float>(argv[6], nq * d);
        const std::string index_path = dir + "/bench.index";

        // Build, as the benchmark does without --cache.
        Index index;
        index = Index(d, nlist, 0, METRIC_L2, OPT_NONE, OPT_ALL, 1, 1, false);
        index.train(nb, base.get());
        index.add(nb, base.get());
        index.save_index(index_path);

        // The --cache path: a default-constructed Index loads the file.
        Index cached;
        cached.load_index(index_path);

        // A worker's copy: centroids received into centroid_codes.get().
        Index worker(d, nlist, 0, METRIC_L2);
        std::memcpy(worker.centroid_codes.get(), index.centroid_codes.get(), nlist * d * sizeof(float));
        worker.add(nb, base.get());

        std::ofstream list0(dir + "/list0.i64", std::ios::binary);
        for (size_t i = 0; i < index.lists[0].get_list_size(); ++i) {
            const int64_t id = static_cast<int64_t>(index.lists[0].candidate_id[i]);
            list0.write(reinterpret_cast<const char*>(&id), sizeof(id));
        }
        list0.close();

        const std::string log_path = dir + "/log.csv";
        for (size_t np : {size_t(1), size_t(4), nlist}) {
            Index* which[3] = {&index, &cached, &worker};
            const char* tag = "abc";
            for (int w = 0; w < 3; ++w) {
                Index& ix = *which[w];
                ix.nprobe = np;
                auto distances = std::make_unique<float[]>(nq * k);
                auto labels = std::make_unique<idx_t[]>(nq * k);
                Index::Param param;
                param.orderOptimize = true;
                param.mode = Index::SearchMode::DIVIDE_GROUP;
                param.pruning = true;
                param.fullWarmUp = false;
                param.groupCount = 2;
                param.teamCount = 2;
                param.teamSize = 4;
                param.hardInBalance = false;
                param.hardInBalanceTeam = 0;
                param.hardInBalanceRatio = 0;
                param.hardInBalanceTeamRatio = 0;
                ix.preSearch(nb, 4, 2, 10, k, &param, dir + "/tmp.index");
                Stats stats = ix.search(nq, query.get(), k, distances.get(), labels.get());
                ix.postSearch();
                stats.nprobe = np;
                stats.recall = 1.0;
                stats.r2 = 1.0;
                stats.worker = 4;
                stats.nb = nb;
                stats.nq = nq;
                stats.d = d;
                stats.k = k;
                stats.mode = Index::to_string(param.mode);
                if (w == 0) stats.myToCsv(log_path, true, "synthetic");
                const std::string sfx = std::to_string(np) + "_" + tag[w];
                write_raw(dir + "/I_" + sfx + ".i64", labels.get(), nq * k);
                write_raw(dir + "/D_" + sfx + ".f32", distances.get(), nq * k);
            }
        }
        write_raw(dir + "/C.f32", index.centroid_codes.get(), nlist * d);
        std::ofstream(dir + "/times.txt") << index.trainTime << " " << index.addTime << " " << index.preSearchTime
                                          << "\n";
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
