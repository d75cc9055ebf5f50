// Layout and arithmetic of the warm-start network, shared by its CUDA kernels
// (csrc/cuda/mlp.cu), the host code that builds its inputs (warm_start.cpp)
// and the FP64 CPU oracle that checks its gradients.
//
// 12 features -> 64 -> 64 -> 3 outputs, GELU (the erf form) after each hidden
// layer. The parameter block (floats) holds, in order: W1 [64][12], b1 [64],
// W2 [64][64], b2 [64], W3 [3][64], b3 [3], then the input normalisation
// (mean [12], scale [12]) applied as (x - mean) * scale before W1; the
// normalisation is set from the training set and not trained.
//
// Outputs: 0 = log(final sigma / stage-one sigma), 1 = log(final gamma /
// stage-one gamma), 2 = log(stage-two objective evaluations).
// Loss: sum over samples and outputs of w_o (y_o - t_o)^2 / 2, divided by the
// number of samples, with w = (1, 1, 0.25).
#pragma once

#include <cstdint>
#include <cstring>

namespace nebula {
namespace mlp {

constexpr int kIn = 12;
constexpr int kHidden = 64;
constexpr int kOut = 3;
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kHidden * kIn;
constexpr int kW2 = kB1 + kHidden;
constexpr int kB2 = kW2 + kHidden * kHidden;
constexpr int kW3 = kB2 + kHidden;
constexpr int kB3 = kW3 + kOut * kHidden;
constexpr int kInMean = kB3 + kOut;
constexpr int kInScale = kInMean + kIn;
constexpr int kParams = kInScale + kIn;  // 5211
constexpr int kTrained = kInMean;        // parameters the optimiser updates

#ifdef __CUDACC__
__host__ __device__
#endif
constexpr float loss_weight(int o) { return o == kOut - 1 ? 0.25f : 1.0f; }

// Inference takes the weight matrices W1, W2, W3 as BF16 values (8-bit
// significand, rounded to nearest even from the FP32 parameters); biases and
// the input normalisation stay FP32, and every sum accumulates in FP32.
// Training updates FP32 parameters.
#ifdef __CUDACC__
__host__ __device__
#endif
inline bool is_weight(int p) {
  return (p >= kW1 && p < kB1) || (p >= kW2 && p < kB2) || (p >= kW3 && p < kB3);
}

#ifdef __CUDACC__
__host__ __device__
#endif
inline float bf16_round(float v) {
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(v);
#else
  std::memcpy(&u, &v, 4);
#endif
  u += 0x7FFFu + ((u >> 16) & 1u);  // finite inputs: round to nearest, ties to even
  u &= 0xFFFF0000u;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float r;
  std::memcpy(&r, &u, 4);
  return r;
#endif
}

}  // namespace mlp
}  // namespace nebula
