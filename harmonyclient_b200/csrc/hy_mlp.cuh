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

// Tensor-core inference.  mlp_pack writes the weights' bf16 operand image
// (mlp_wimg_bytes() bytes) from the parameter vector; mlp_infer computes, for
// m queries with their P best coarse scores (pscore, m x P, best first), the
// standardised features, the network output y (into yout when given) and,
// when probes (m x P) is given, cuts each query's probes past
// clamp(ceil(2^(y + margin)), 1, P) to -1 and adds the kept counts to *total.
size_t mlp_wimg_bytes();
cudaError_t mlp_pack(const float* params, unsigned char* wimg, cudaStream_t s);
cudaError_t mlp_infer(const float* pscore, int m, int P, const float* mu, const float* sd, const unsigned char* wimg,
                      const float* params, float margin, int64_t* probes, unsigned long long* total, float* yout,
                      int* err, cudaStream_t s);

}  // namespace hy
