// Stand-in for faiss/IndexFlat.h used only when compiling the reference's
// Index.cpp into the oracle library.  The reference uses faiss solely in
// Index::train(..., faiss=true), which the oracle never calls; the vendored
// faiss needs BLAS/LAPACK to build, so these classes exist only to satisfy
// the compiler and throw if constructed.
#pragma once
#include <cstddef>
#include <stdexcept>
#include <faiss/MetricType.h>
namespace faiss {
struct Index {};
struct IndexFlatL2 : Index {
    explicit IndexFlatL2(long) { throw std::runtime_error("faiss training is not built into the oracle"); }
    const float* get_xb() const { return nullptr; }
};
}  // namespace faiss
