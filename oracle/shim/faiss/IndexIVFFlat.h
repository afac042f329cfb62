// Stand-in for faiss/IndexIVFFlat.h; see IndexFlat.h in this directory.
#pragma once
#include "IndexFlat.h"
namespace faiss {
struct IndexIVFFlat : Index {
    IndexIVFFlat(Index*, size_t, size_t) { throw std::runtime_error("faiss training is not built into the oracle"); }
    void train(long, const float*) {}
};
}  // namespace faiss
