// The probe-predictor network (hy_mlp.cu): shapes, parameter layout and the
// launchers used by the index's training and search.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace hy {

constexpr int MLP_IN = 64;    // sorted centroid-distance features
constexpr int MLP_H = 256;    // hidden width (two hidden layers)
constexpr int MLP_W1 = 0;
constexpr int MLP_B1 = MLP_W1 + MLP_IN * MLP_H;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_H;
constexpr int MLP_NPARAM = MLP_B3 + 1;

// Activation buffers of one batch of B rows (each B x MLP_H floats).
struct MlpWork {
    float *Z1, *A1, *Z2, *A2, *dA, *dZ;
};
size_t mlp_work_floats(int B);
void mlp_work_bind(MlpWork& w, float* base, int B);

cudaError_t mlp_forward(const float* params, int B, const float* X, MlpWork& w, float* y, cudaStream_t s);
cudaError_t mlp_backward(const float* params, int B, const float* X, MlpWork& w, const float* dy, float* grads,
                         cudaStream_t s);
cudaError_t mlp_mse(int B, const float* y, const float* t, float* dy, float* loss, cudaStream_t s);
cudaError_t mlp_adam(float* params, const float* grads, float* m, float* v, int step, float lr, cudaStream_t s);

}  // namespace hy
