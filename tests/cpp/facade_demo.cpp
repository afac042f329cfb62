// Uses the harmony::Index facade exactly as the reference's callers use
// harmony::Index (src/main.cpp:48-71, src/query.cpp:833-934): construct,
// train, add, preSearch, search.  Reads base and queries as raw float32 files,
// writes distances and labels as raw files.
//   facade_demo <d> <nlist> <nprobe> <k> <base.f32> <nb> <queries.f32> <nq> <out_prefix> [bf16]
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "harmony/Index.h"

static std::vector<float> read_f32(const char* path, size_t n) {
    std::vector<float> v(n);
    std::ifstream in(path, std::ios::binary);
    in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(n * sizeof(float)));
    if (!in) throw std::runtime_error(std::string("cannot read ") + path);
    return v;
}

int main(int argc, char** argv) {
    if (argc < 10) {
        std::fprintf(stderr, "usage: facade_demo d nlist nprobe k base nb queries nq out_prefix [bf16]\n");
        return 2;
    }
    const size_t d = std::strtoul(argv[1], nullptr, 10), nlist = std::strtoul(argv[2], nullptr, 10);
    const size_t nprobe = std::strtoul(argv[3], nullptr, 10), k = std::strtoul(argv[4], nullptr, 10);
    const size_t nb = std::strtoul(argv[6], nullptr, 10), nq = std::strtoul(argv[8], nullptr, 10);
    try {
        auto base = read_f32(argv[5], nb * d);
        auto q = read_f32(argv[7], nq * d);
        harmony::Index index(d, nlist, nprobe, harmony::METRIC_L2, harmony::OPT_NONE, harmony::OPT_ALL);
        if (argc > 10) index.set_form(HY_FORM_BF16);
        index.train(nb, base.data());
        index.add(nb, base.data());
        harmony::Index::Param param;
        index.preSearch(nb, 1, 1, 10, k, &param, "");
        std::vector<float> D(nq * k);
        std::vector<harmony::idx_t> I(nq * k);
        harmony::Stats st = index.search(nq, q.data(), k, D.data(), I.data());
        std::string pre = argv[9];
        std::ofstream(pre + ".D", std::ios::binary).write(reinterpret_cast<const char*>(D.data()), D.size() * 4);
        std::ofstream(pre + ".I", std::ios::binary).write(reinterpret_cast<const char*>(I.data()), I.size() * 8);
        std::ofstream(pre + ".C", std::ios::binary)
            .write(reinterpret_cast<const char*>(index.centroid_codes.get()), nlist * d * 4);
        std::cout << "searched " << st.nq << " queries, skip rate " << st.skip_rate() << "\n";
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
