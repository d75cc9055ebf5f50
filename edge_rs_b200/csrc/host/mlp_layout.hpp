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

}  // namespace mlp
}  // namespace nebula
