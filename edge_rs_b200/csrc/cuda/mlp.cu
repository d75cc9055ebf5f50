// The warm-start network on the GPU: inference, the loss gradient and Adam
// training, with the project's own kernels (layout and loss in
// ../host/mlp_layout.hpp).
//
// Gradient: a tile of 64 samples per pass of a CTA; 64 threads run one
// sample's forward and backward pass each and leave its normalised inputs,
// activations and deltas in shared memory, then all 256 threads form the
// parameter gradients as sums over the tile's samples in sample order. Each
// CTA keeps its partial sums in registers across tiles and writes them out;
// a second kernel adds the CTAs' partials in CTA order. No atomics, so a
// gradient (and a training run) is bitwise reproducible.
//
// Training: one Adam step is four kernels (gradient, reduction, update,
// cursor advance) that read the mini-batch position and the step count from
// device memory; they are captured once in a CUDA graph and the graph is
// launched once per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../host/common.hpp"
#include "../host/export.hpp"
#include "../host/mlp_layout.hpp"

namespace nebula {
namespace device {
namespace {

using namespace mlp;

constexpr int kTile = 64;           // samples per tile
constexpr int kMlpThreads = 256;
constexpr int kRow = kIn + 4 * kHidden + kOut;  // per-sample row in shared memory (271, odd)
constexpr int kSlots = (kTrained + kMlpThreads - 1) / kMlpThreads;
constexpr int kMaxGradBlocks = 64;
// row layout
constexpr int kRx = 0, kRh1 = kIn, kRh2 = kRh1 + kHidden, kRd1 = kRh2 + kHidden, kRd2 = kRd1 + kHidden,
              kRd3 = kRd2 + kHidden;

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Forward pass of one sample; `row` (shared memory) receives the normalised
// inputs, both hidden activations and, in the delta slots, the GELU
// derivatives at the pre-activations. Returns the outputs in y.
__device__ void forward_row(const float* w, const float* x, float* row, float* y) {
  for (int k = 0; k < kIn; ++k) row[kRx + k] = (x[k] - w[kInMean + k]) * w[kInScale + k];
  for (int i = 0; i < kHidden; ++i) {
    float a = w[kB1 + i];
    for (int k = 0; k < kIn; ++k) a = fmaf(w[kW1 + i * kIn + k], row[kRx + k], a);
    row[kRh1 + i] = gelu(a);
    row[kRd1 + i] = gelu_grad(a);
  }
  for (int i = 0; i < kHidden; ++i) {
    float a = w[kB2 + i];
    for (int j = 0; j < kHidden; ++j) a = fmaf(w[kW2 + i * kHidden + j], row[kRh1 + j], a);
    row[kRh2 + i] = gelu(a);
    row[kRd2 + i] = gelu_grad(a);
  }
  for (int o = 0; o < kOut; ++o) {
    float a = w[kB3 + o];
    for (int h = 0; h < kHidden; ++h) a = fmaf(w[kW3 + o * kHidden + h], row[kRh2 + h], a);
    y[o] = a;
  }
}

__global__ void __launch_bounds__(kMlpThreads) mlp_predict_kernel(const float* __restrict__ params,
                                                                  const float* __restrict__ features, int n,
                                                                  float* __restrict__ out) {
  extern __shared__ float sh[];
  float* w = sh;
  float* rows = sh + kParams;
  // the weights as BF16 values (mlp_layout.hpp), FP32 accumulation
  for (int p = threadIdx.x; p < kParams; p += blockDim.x) w[p] = is_weight(p) ? bf16_round(params[p]) : params[p];
  __syncthreads();
  for (int base = blockIdx.x * kTile; base < n; base += gridDim.x * kTile) {
    const int s = base + static_cast<int>(threadIdx.x);
    if (threadIdx.x < kTile && s < n) {
      float y[kOut];
      forward_row(w, features + static_cast<size_t>(s) * kIn, rows + threadIdx.x * kRow, y);
      for (int o = 0; o < kOut; ++o) out[static_cast<size_t>(s) * kOut + o] = y[o];
    }
  }
}

// Partial gradient of the loss over rows perm[cursor .. cursor + batch) (or
// rows cursor .. when perm is null), clipped to n; inv_n scales the loss
// (1 / the batch's sample count). partial: gridDim.x x kTrained,
// partial_loss: gridDim.x.
__global__ void __launch_bounds__(kMlpThreads) mlp_grad_kernel(const float* __restrict__ params,
                                                               const float* __restrict__ features,
                                                               const float* __restrict__ targets,
                                                               const int* __restrict__ perm,
                                                               const int* __restrict__ cursor, int batch, int n,
                                                               float* __restrict__ partial,
                                                               double* __restrict__ partial_loss) {
  extern __shared__ float sh[];
  float* w = sh;
  float* rows = sh + kParams;
  __shared__ float loss_of[kTile];
  for (int p = threadIdx.x; p < kParams; p += blockDim.x) w[p] = params[p];
  const int start = cursor ? *cursor : 0;
  const int count = min(batch, n - start);
  const float inv_n = count > 0 ? 1.0f / static_cast<float>(count) : 0.0f;
  float acc[kSlots];
#pragma unroll
  for (int k = 0; k < kSlots; ++k) acc[k] = 0.0f;
  double block_loss = 0.0;
  __syncthreads();
  for (int base = blockIdx.x * kTile; base < count; base += gridDim.x * kTile) {
    const int tid = threadIdx.x;
    if (tid < kTile) {
      float* row = rows + tid * kRow;
      const int s = base + tid;
      if (s < count) {
        const int r = perm ? perm[start + s] : start + s;
        float y[kOut];
        forward_row(w, features + static_cast<size_t>(r) * kIn, row, y);
        float d3[kOut];
        float l = 0.0f;
        for (int o = 0; o < kOut; ++o) {
          const float e = y[o] - targets[static_cast<size_t>(r) * kOut + o];
          l += loss_weight(o) * e * e * 0.5f;
          d3[o] = loss_weight(o) * e * inv_n;
          row[kRd3 + o] = d3[o];
        }
        loss_of[tid] = l;
        for (int h = 0; h < kHidden; ++h) {
          float g = 0.0f;
          for (int o = 0; o < kOut; ++o) g = fmaf(w[kW3 + o * kHidden + h], d3[o], g);
          row[kRd2 + h] *= g;
        }
        for (int i = 0; i < kHidden; ++i) {
          float g = 0.0f;
          for (int h = 0; h < kHidden; ++h) g = fmaf(w[kW2 + h * kHidden + i], row[kRd2 + h], g);
          row[kRd1 + i] *= g;
        }
      } else {
        for (int c = 0; c < kRow; ++c) row[c] = 0.0f;
        loss_of[tid] = 0.0f;
      }
    }
    __syncthreads();
    if (tid == 0)
      for (int s = 0; s < kTile; ++s) block_loss += static_cast<double>(loss_of[s]);
    // parameter gradients: sums over the tile's samples, in sample order
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      const int p = tid + k * kMlpThreads;
      if (p >= kTrained) break;
      float g = 0.0f;
      if (p < kB1) {
        const int i = p / kIn, c = p - i * kIn;
        for (int s = 0; s < kTile; ++s) g = fmaf(rows[s * kRow + kRd1 + i], rows[s * kRow + kRx + c], g);
      } else if (p < kW2) {
        const int i = p - kB1;
        for (int s = 0; s < kTile; ++s) g += rows[s * kRow + kRd1 + i];
      } else if (p < kB2) {
        const int q = p - kW2, i = q / kHidden, j = q - i * kHidden;
        for (int s = 0; s < kTile; ++s) g = fmaf(rows[s * kRow + kRd2 + i], rows[s * kRow + kRh1 + j], g);
      } else if (p < kW3) {
        const int i = p - kB2;
        for (int s = 0; s < kTile; ++s) g += rows[s * kRow + kRd2 + i];
      } else if (p < kB3) {
        const int q = p - kW3, o = q / kHidden, h = q - o * kHidden;
        for (int s = 0; s < kTile; ++s) g = fmaf(rows[s * kRow + kRd3 + o], rows[s * kRow + kRh2 + h], g);
      } else {
        const int o = p - kB3;
        for (int s = 0; s < kTile; ++s) g += rows[s * kRow + kRd3 + o];
      }
      acc[k] += g;
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < kSlots; ++k) {
    const int p = threadIdx.x + k * kMlpThreads;
    if (p < kTrained) partial[static_cast<size_t>(blockIdx.x) * kTrained + p] = acc[k];
  }
  if (threadIdx.x == 0) partial_loss[blockIdx.x] = block_loss * static_cast<double>(inv_n);
}

// grad[p] = sum over blocks of partial[b][p] in block order; thread 0 also
// adds the batch loss to *loss_sum.
__global__ void mlp_reduce_kernel(const float* __restrict__ partial, const double* __restrict__ partial_loss,
                                  int blocks, float* __restrict__ grad, double* __restrict__ loss_sum) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kTrained) {
    float g = 0.0f;
    for (int b = 0; b < blocks; ++b) g += partial[static_cast<size_t>(b) * kTrained + p];
    grad[p] = g;
  }
  if (p == 0 && loss_sum) {
    double l = 0.0;
    for (int b = 0; b < blocks; ++b) l += partial_loss[b];
    *loss_sum += l;
  }
}

// One Adam step (Kingma and Ba, 2015) on the trained parameters; step[0] is
// the number of steps taken before this one.
__global__ void mlp_adam_kernel(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m,
                                float* __restrict__ v, const int* __restrict__ step, float lr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kTrained) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int t = *step + 1;
  const float g = grad[p];
  const float mp = b1 * m[p] + (1.0f - b1) * g;
  const float vp = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mp;
  v[p] = vp;
  const float mh = mp / (1.0f - powf(b1, static_cast<float>(t)));
  const float vh = vp / (1.0f - powf(b2, static_cast<float>(t)));
  params[p] -= lr * mh / (sqrtf(vh) + eps);
}

// Moves the mini-batch cursor and counts the step (one thread).
__global__ void mlp_advance_kernel(int* cursor, int* step, int batch, int n) {
  const int next = *cursor + batch;
  *cursor = next >= n ? 0 : next;
  *step += 1;
}

size_t grad_smem() { return (static_cast<size_t>(kParams) + static_cast<size_t>(kTile) * kRow) * sizeof(float); }

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(NB_ERR_GPU, std::string(what) + ": " + cudaGetErrorString(e));
}

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  const size_t n = std::min(len - 1, msg.size());
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

template <typename T>
struct DeviceBuffer {
  T* ptr = nullptr;
  explicit DeviceBuffer(size_t n) { check(cudaMalloc(reinterpret_cast<void**>(&ptr), std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc"); }
  ~DeviceBuffer() {
    if (ptr) cudaFree(ptr);
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  void upload(const T* host, size_t n) {
    if (n) check(cudaMemcpy(ptr, host, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  }
  void download(T* host, size_t n) const {
    if (n) check(cudaMemcpy(host, ptr, n * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
  }
};

void configure() {
  check(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(grad_smem())),
        "mlp attribute");
  check(cudaFuncSetAttribute(mlp_predict_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(grad_smem())),
        "mlp attribute");
}

int grad_blocks(int count) { return std::max(1, std::min(kMaxGradBlocks, (count + kTile - 1) / kTile)); }

// xorshift64* (Vigna, 2016), for initial weights and epoch shuffles
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ULL + 0x2545F4914F6CDD1DULL) {
    if (!s) s = 1;
  }
  uint64_t next() {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    return s * 0x2545F4914F6CDD1DULL;
  }
  double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace
}  // namespace device
}  // namespace nebula

using nebula::NbError;
using nebula::fail;
namespace dv = nebula::device;
namespace ml = nebula::mlp;

// Xavier-uniform initial weights (deterministic in `seed`), zero biases,
// identity input normalisation.
NB_API void nb_mlp_init(uint64_t seed, float* params) {
  dv::Rng rng(seed);
  auto fill = [&](int off, int rows, int cols) {
    const double a = std::sqrt(6.0 / static_cast<double>(rows + cols));
    for (int i = 0; i < rows * cols; ++i) params[off + i] = static_cast<float>((2.0 * rng.uniform() - 1.0) * a);
  };
  std::fill(params, params + ml::kParams, 0.0f);
  fill(ml::kW1, ml::kHidden, ml::kIn);
  fill(ml::kW2, ml::kHidden, ml::kHidden);
  fill(ml::kW3, ml::kOut, ml::kHidden);
  for (int k = 0; k < ml::kIn; ++k) params[ml::kInScale + k] = 1.0f;
}

NB_API int32_t nb_mlp_predict_cuda(const float* params, const float* features, uint64_t n, float* out, char* err,
                                   size_t err_len) {
  try {
    if (!params || (n && (!features || !out))) fail(NB_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return NB_OK;
    if (n > (1ULL << 30)) fail(NB_ERR_INVALID_ARGUMENT, "too many samples");
    dv::configure();
    dv::DeviceBuffer<float> p(ml::kParams), x(n * ml::kIn), y(n * ml::kOut);
    p.upload(params, ml::kParams);
    x.upload(features, n * ml::kIn);
    const int blocks = static_cast<int>(std::min<uint64_t>((n + dv::kTile - 1) / dv::kTile, 1024));
    dv::mlp_predict_kernel<<<blocks, dv::kMlpThreads, dv::grad_smem()>>>(p.ptr, x.ptr, static_cast<int>(n), y.ptr);
    dv::check(cudaGetLastError(), "mlp predict launch");
    y.download(out, n * ml::kOut);
    return NB_OK;
  } catch (const NbError& e) {
    dv::write_err(err, err_len, e.message);
    return e.code;
  }
}

NB_API int32_t nb_mlp_gradient_cuda(const float* params, const float* features, const float* targets, uint64_t n,
                                    float* grad_out, double* loss_out, char* err, size_t err_len) {
  try {
    if (!params || !grad_out || n == 0 || !features || !targets) fail(NB_ERR_INVALID_ARGUMENT, "null or empty argument");
    if (n > (1ULL << 30)) fail(NB_ERR_INVALID_ARGUMENT, "too many samples");
    dv::configure();
    const int count = static_cast<int>(n);
    const int blocks = dv::grad_blocks(count);
    dv::DeviceBuffer<float> p(ml::kParams), x(n * ml::kIn), t(n * ml::kOut), part(blocks * ml::kTrained),
        g(ml::kTrained);
    dv::DeviceBuffer<double> pl(blocks), loss(1);
    p.upload(params, ml::kParams);
    x.upload(features, n * ml::kIn);
    t.upload(targets, n * ml::kOut);
    dv::check(cudaMemset(loss.ptr, 0, sizeof(double)), "memset");
    dv::mlp_grad_kernel<<<blocks, dv::kMlpThreads, dv::grad_smem()>>>(p.ptr, x.ptr, t.ptr, nullptr, nullptr, count,
                                                                      count, part.ptr, pl.ptr);
    dv::check(cudaGetLastError(), "mlp gradient launch");
    dv::mlp_reduce_kernel<<<(ml::kTrained + 255) / 256, 256>>>(part.ptr, pl.ptr, blocks, g.ptr, loss.ptr);
    dv::check(cudaGetLastError(), "mlp reduce launch");
    std::vector<float> host(ml::kTrained);
    g.download(host.data(), ml::kTrained);
    std::copy(host.begin(), host.end(), grad_out);
    std::fill(grad_out + ml::kTrained, grad_out + ml::kParams, 0.0f);
    if (loss_out) loss.download(loss_out, 1);
    return NB_OK;
  } catch (const NbError& e) {
    dv::write_err(err, err_len, e.message);
    return e.code;
  }
}

NB_API int32_t nb_mlp_train_cuda(const float* features, const float* targets, uint64_t n, int32_t epochs,
                                 int32_t batch, float lr, uint64_t seed, float* params, double* epoch_loss,
                                 char* err, size_t err_len) {
  try {
    if (!params || !features || !targets || n == 0) fail(NB_ERR_INVALID_ARGUMENT, "null or empty argument");
    if (n > (1ULL << 30)) fail(NB_ERR_INVALID_ARGUMENT, "too many samples");
    if (epochs < 1 || batch < 1) fail(NB_ERR_MUST_BE_POSITIVE, "epochs and batch must be positive");
    if (!(lr > 0.0f)) fail(NB_ERR_MUST_BE_POSITIVE, "the learning rate must be positive");
    dv::configure();
    const int count = static_cast<int>(n);
    const int b = std::min(batch, count);
    const int blocks = dv::grad_blocks(b);
    dv::DeviceBuffer<float> p(ml::kParams), x(n * ml::kIn), t(n * ml::kOut), part(blocks * ml::kTrained),
        g(ml::kTrained), m(ml::kTrained), v(ml::kTrained);
    dv::DeviceBuffer<double> pl(blocks), losses(epochs);
    dv::DeviceBuffer<int> perm(n), state(2);  // state: cursor, step
    p.upload(params, ml::kParams);
    x.upload(features, n * ml::kIn);
    t.upload(targets, n * ml::kOut);
    dv::check(cudaMemset(m.ptr, 0, ml::kTrained * sizeof(float)), "memset");
    dv::check(cudaMemset(v.ptr, 0, ml::kTrained * sizeof(float)), "memset");
    dv::check(cudaMemset(state.ptr, 0, 2 * sizeof(int)), "memset");
    dv::check(cudaMemset(losses.ptr, 0, epochs * sizeof(double)), "memset");
    cudaStream_t stream = nullptr;
    dv::check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaGraphExec_t exec = nullptr;
    auto cleanup = [&]() {
      if (exec) cudaGraphExecDestroy(exec);
      if (stream) cudaStreamDestroy(stream);
    };
    try {
      // the four kernels of one step are captured once per epoch (the
      // epoch's loss slot is their one changing argument) and the graph is
      // launched once per step
      const int steps = (count + b - 1) / b;
      std::vector<int> order(n);
      dv::Rng rng(seed);
      for (int e = 0; e < epochs; ++e) {
        for (int i = 0; i < count; ++i) order[i] = i;
        for (int i = count - 1; i > 0; --i) std::swap(order[i], order[static_cast<int>(rng.next() % (i + 1))]);
        // the previous epoch's steps still read the permutation
        dv::check(cudaStreamSynchronize(stream), "training");
        perm.upload(order.data(), n);
        cudaGraph_t graph = nullptr;
        dv::check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
        dv::mlp_grad_kernel<<<blocks, dv::kMlpThreads, dv::grad_smem(), stream>>>(
            p.ptr, x.ptr, t.ptr, perm.ptr, state.ptr, b, count, part.ptr, pl.ptr);
        dv::mlp_reduce_kernel<<<(ml::kTrained + 255) / 256, 256, 0, stream>>>(part.ptr, pl.ptr, blocks, g.ptr,
                                                                              losses.ptr + e);
        dv::mlp_adam_kernel<<<(ml::kTrained + 255) / 256, 256, 0, stream>>>(p.ptr, g.ptr, m.ptr, v.ptr,
                                                                            state.ptr + 1, lr);
        dv::mlp_advance_kernel<<<1, 1, 0, stream>>>(state.ptr, state.ptr + 1, b, count);
        dv::check(cudaStreamEndCapture(stream, &graph), "capture end");
        if (exec) {
          cudaGraphExecDestroy(exec);
          exec = nullptr;
        }
        const cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        dv::check(inst, "graph instantiate");
        for (int s = 0; s < steps; ++s) dv::check(cudaGraphLaunch(exec, stream), "graph launch");
      }
      dv::check(cudaStreamSynchronize(stream), "training");
    } catch (...) {
      cudaStreamSynchronize(stream);
      cleanup();
      throw;
    }
    cleanup();
    p.download(params, ml::kParams);
    if (epoch_loss) {
      std::vector<double> l(epochs);
      losses.download(l.data(), epochs);
      const int steps = (count + b - 1) / b;
      for (int e = 0; e < epochs; ++e) epoch_loss[e] = l[e] / steps;  // mean batch loss of the epoch
    }
    return NB_OK;
  } catch (const NbError& e) {
    dv::write_err(err, err_len, e.message);
    return e.code;
  }
}
