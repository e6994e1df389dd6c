// lfsai.cuh -- constants and handle of the learned FSAI network.
#pragma once

#include "internal.cuh"

namespace tnlb {

// Network 32 -> 64 -> 64 -> 64 -> 8 and its parameter layout (FP32 master):
// W1 (64x32 row-major), b1, W2 (64x64), b2, W3, b3, W4 (8x64), b4.  Up to
// kLfK = 8 entries per row of G; kLfPairs features from the slot pairs.
constexpr int kLfF = 32, kLfH = 64, kLfK = 8, kLfPairs = kLfK * (kLfK - 1) / 2;
constexpr int kLfW1 = 0;
constexpr int kLfB1 = kLfW1 + kLfH * kLfF;
constexpr int kLfW2 = kLfB1 + kLfH;
constexpr int kLfB2 = kLfW2 + kLfH * kLfH;
constexpr int kLfW3 = kLfB2 + kLfH;
constexpr int kLfB3 = kLfW3 + kLfH * kLfH;
constexpr int kLfW4 = kLfB3 + kLfH;
constexpr int kLfB4 = kLfW4 + kLfK * kLfH;
constexpr int kLfParams = kLfB4 + kLfK;
static_assert(kLfParams == 10952, "parameter layout");
static_assert(kLfPairs + 4 == kLfF, "feature layout");

}  // namespace tnlb

// Network parameters and Adam state (opaque in the C ABI).
struct tnlb_lfsai {
   tnlb::DeviceBuffer theta;   // FP32 master parameters
   tnlb::DeviceBuffer wround;  // BF16-rounded weights (biases FP32) used by the forward pass
   tnlb::DeviceBuffer grad;    // FP32 gradient of the last step
   tnlb::DeviceBuffer m, v;    // Adam moments
   int64_t step = 0;
   int use_tc = 1;             // dense layers on tcgen05 tensor cores (else CUDA cores)
   int level = 1;              // pattern of G: 0 lower triangle of A, 1 of A^2
   int two_factor = 0;         // nonsymmetric A: G_L and H = G_U^T on the level-0 pattern
};

namespace tnlb {
tnlb_status lfsai_init(tnlb_lfsai* net, uint64_t seed, cudaStream_t st);
tnlb_status lfsai_forward(const tnlb_lfsai* net, const float* feat, int64_t n, float* o, float* h1, float* h2,
                          float* h3, cudaStream_t st);
// mode: 0 probe loss, 1 warm-start regression, 2 Kaporin loss
tnlb_status lfsai_gradient(tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                           const void* vals, const void* probes, int32_t P, int mode, cudaStream_t st, double* loss);
tnlb_status lfsai_adam(tnlb_lfsai* net, double lr, cudaStream_t st);
tnlb_status lfsai_precond(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                          const void* vals, cudaStream_t st, tnlb_precond** out);
tnlb_status lfsai_forward_tc(const tnlb_lfsai* net, const float* feat, int64_t n, float* o, float* h1, float* h2,
                             float* h3, cudaStream_t st);
// Backward through the layers on tcgen05: d3, d2, d1 (n x 64, FP32) from
// dL/do, then the weight and bias gradients into net->grad.
tnlb_status lfsai_backward_tc(tnlb_lfsai* net, const float* feat, int64_t n, const float* h1, const float* h2,
                              const float* h3, const float* dout, cudaStream_t st);
tnlb_status lfsai_eval(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                       const void* vals, cudaStream_t st, float* h_feat, float* h_out);
}  // namespace tnlb
