// lfsai.cuh -- constants and handle of the learned FSAI network.
#pragma once

#include "internal.cuh"

namespace tnlb {

// Network 16 -> 64 -> 64 -> 64 -> 4 and its parameter layout (FP32 master):
// W1 (64x16 row-major), b1, W2 (64x64), b2, W3, b3, W4 (4x64), b4.
constexpr int kLfF = 16, kLfH = 64, kLfK = 4;
constexpr int kLfW1 = 0;
constexpr int kLfB1 = kLfW1 + kLfH * kLfF;
constexpr int kLfW2 = kLfB1 + kLfH;
constexpr int kLfB2 = kLfW2 + kLfH * kLfH;
constexpr int kLfW3 = kLfB2 + kLfH;
constexpr int kLfB3 = kLfW3 + kLfH * kLfH;
constexpr int kLfW4 = kLfB3 + kLfH;
constexpr int kLfB4 = kLfW4 + kLfK * kLfH;
constexpr int kLfParams = kLfB4 + kLfK;
static_assert(kLfParams == 9668, "parameter layout");

}  // namespace tnlb

// Network parameters and Adam state (opaque in the C ABI).
struct tnlb_lfsai {
   tnlb::DeviceBuffer theta;   // FP32 master parameters
   tnlb::DeviceBuffer wround;  // BF16-rounded weights (biases FP32) used by the forward pass
   tnlb::DeviceBuffer grad;    // FP32 gradient of the last step
   tnlb::DeviceBuffer m, v;    // Adam moments
   int64_t step = 0;
   int use_tc = 0;             // dense layers on tcgen05 tensor cores
};

namespace tnlb {
tnlb_status lfsai_init(tnlb_lfsai* net, uint64_t seed, cudaStream_t st);
tnlb_status lfsai_forward(const tnlb_lfsai* net, const float* feat, int64_t n, float* o, float* h1, float* h2,
                          float* h3, cudaStream_t st);
tnlb_status lfsai_gradient(tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                           const void* vals, const void* probes, int32_t P, bool fit, cudaStream_t st, double* loss);
tnlb_status lfsai_adam(tnlb_lfsai* net, double lr, cudaStream_t st);
tnlb_status lfsai_precond(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                          const void* vals, cudaStream_t st, tnlb_precond** out);
tnlb_status lfsai_forward_tc(const tnlb_lfsai* net, const float* feat, int64_t n, float* o, float* h1, float* h2,
                             float* h3, cudaStream_t st);
tnlb_status lfsai_eval(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                       const void* vals, cudaStream_t st, float* h_feat, float* h_out);
}  // namespace tnlb
