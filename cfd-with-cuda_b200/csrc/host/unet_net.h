// Host side of the learned pressure preconditioner: the U-Net's layer list,
// its parameters (FP32 master copy, BF16 copy for the kernels, Adam moments),
// activation and gradient buffers, and the forward / backward / training
// drivers that launch the kernels of unet.cu.
//
// Layer list (grids L0 = nx x ny x nz pressure nodes, L1 and L2 every other
// node of the level above, so each axis needs (n - 1) % 4 == 0):
//   t0  x      1 ch  L0   network input (unit-RMS residual)
//   c0  t0 -> t1   1 -> 16 L0        3x3x3 conv, act
//   c1  t1 -> t2  16 -> 32 L0 -> L1  stride-2 conv, act
//   c2  t2 -> t3  32 -> 32 L1        conv, act
//   c3  t3 -> t4  32 -> 64 L1 -> L2  stride-2 conv, act
//   c4  t4 -> t5  64 -> 64 L2        conv, act
//   c5  t5 -> t6  64 -> 64 L2        conv, act
//   c6  t6 -> t7  64 -> 32 L2        conv, act
//   u0  t8 = P(t7) + t3     32 ch L1 prolongation plus skip
//   c7  t8 -> t9  32 -> 32 L1        conv, act
//   c8  t9 -> t10 32 -> 16 L1        conv, act
//   u1  t11 = P(t10) + t1   16 ch L0
//   c9  t11 -> t12 16 -> 16 L0       conv, act
//   c10 t12 -> t13 16 -> 1  L0       conv, FP32 output (the correction)
// act = leaky ReLU (slope 0.1).  Weights [27][cin][cout] with tap
// k = (dx+1) + 3 (dy+1) + 9 (dz+1), then the bias [cout], layer after layer.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../cuda/unet.h"

#include <cstdint>
#include <string>
#include <vector>

namespace cfd {

constexpr int kUnetConvs = 11;
constexpr int kUnetTensors = 14;

struct UnetConvSpec {
  int in, out, stride, act;
};
struct UnetUpSpec {
  int in, skip, out;
};
struct UnetTensorSpec {
  int level, ch;
};
extern const UnetConvSpec kUnetConv[kUnetConvs];
extern const UnetUpSpec kUnetUp[2];
extern const UnetTensorSpec kUnetTensor[kUnetTensors];

// Parameter count and per-layer offsets (weights, then bias) of the list above.
long long unet_param_count();
long long unet_weight_offset(int layer);
long long unet_bias_offset(int layer);

struct UnetNet {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  long long nparam = 0;
  float *P = nullptr, *G = nullptr, *M1 = nullptr, *M2 = nullptr;  // master params, grads, Adam moments
  __nv_bfloat16* Pb = nullptr;                                      // BF16 copy of P
  int adam_t = 0;
  float w_l2 = 1.f, w_h1 = 0.f;  // training loss weights (unet_loss)
  long long launches = 0;
  std::string err;

  // activations sized for the largest grid seen so far
  int dims[3][3] = {};
  long long nvox[3] = {0, 0, 0};
  long long cap[kUnetTensors] = {};
  __nv_bfloat16* act[kUnetTensors] = {};
  float* out = nullptr;  // t13 (FP32)
  long long out_cap = 0;
  float* grad[kUnetTensors] = {};
  long long gcap[kUnetTensors] = {};
  float* lossv = nullptr;
  float* h_pinned = nullptr;
  int gen = 0;  // bumped whenever an activation buffer moves

  // tensor-core path: packed weights and launch plans of the stride-1 layers
  bool tc_enabled = true;
  // tensor-core kernel of each layer (CFD_CONV_PIPE): 0 one CTA per brick;
  // 1 the persistent kernel; 2 the persistent kernel with the dx taps folded
  // on the stride-1 layers, one CTA per brick on the stride-2 layers; 3 as 2
  // with the persistent kernel on the stride-2 layers
  int conv_pipe = 0;
  // conv_tc_plan's pipe argument for a layer of this stride
  int pipe_mode(int stride) const {
    if (stride == 1) return conv_pipe == 1 ? 1 : (conv_pipe >= 2 ? 2 : 0);
    return conv_pipe == 1 || conv_pipe == 3 ? 1 : 0;
  }
  int num_sms = 148;
  __nv_bfloat16* wpack[kUnetConvs] = {};
  long long wpack_cap[kUnetConvs] = {};
  bool packs_dirty = true;
  ConvTcPlan plans[kUnetConvs];
  bool plan_ok[kUnetConvs] = {};
  int plan_gen = -1, plan_dims[3] = {0, 0, 0};
  int* tc_err = nullptr;

  ~UnetNet();
  // Allocates parameters on the current device and initialises them from seed.
  int init(unsigned long long seed);
  // Host copy in / out of the FP32 parameters (refreshes the BF16 copy).
  int set_params(const float* h, long long n);
  int get_params(float* h, long long n);
  // Sets the grid and (re)allocates activations; train != 0 also gradients.
  int set_grid(const int d[3], bool train);
  // Packs weights and builds plans for the tensor-core layers when needed.
  cudaError_t prepare_tc(cudaStream_t s);
  // Forward pass of the grid set by set_grid: act[0] must hold the input;
  // writes the FP32 output to out_f32 (or this->out when null).  Every
  // kernel is a no-op while the device flag *skip is set (skip may be null).
  cudaError_t forward(cudaStream_t s, float* out_f32, const int* skip = nullptr);
  // Backward pass from grad of the output (in grad[13]); accumulates
  // parameter gradients into G (not zeroed here).
  cudaError_t backward(cudaStream_t s);
  // One optimiser step on accumulated gradients, scaled by gscale.
  cudaError_t adam(cudaStream_t s, float lr, float gscale);
};

}  // namespace cfd
