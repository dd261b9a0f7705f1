// Learned pressure preconditioner: a 3-level 3D convolutional U-Net on the
// structured grid of pressure nodes (hand-written CUDA forward and backward
// kernels; BF16 weights and activations, FP32 accumulation and gradients).
//
// Grid levels: L0 = (nx, ny, nz) pressure nodes, L1 = ((n-1)/2 + 1) per axis
// (every other node), L2 likewise.  Activations are channels-last
// (voxel-major, channels contiguous), voxel v = x + nx (y + ny z).
//
// The layer list lives in the host network (unet_net.h); these are its
// building blocks.  Activation: leaky ReLU, slope 0.1.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cfd {

constexpr float kLeaky = 0.1f;

struct ConvDesc {
  int in_dims[3], out_dims[3];
  int stride;                 // 1 or 2
  const __nv_bfloat16* inA;   // channels-last, ca channels
  int ca;
  const __nv_bfloat16* inB;   // optional second input (concatenated channels), cb channels
  int cb;
  int cout;
  const __nv_bfloat16* w;     // [27][ca+cb][cout]
  const float* bias;          // [cout]
  __nv_bfloat16* out;         // bf16 output (or null)
  float* out_f32;             // FP32 output (or null)
  int act;                    // 1: leaky ReLU
  const int* skip;            // optional device flag: the kernel does nothing while *skip != 0
};

cudaError_t conv3_forward(const ConvDesc& d, cudaStream_t s);

// dIn = conv^T(dOut, W): writes FP32 gradients of inA (dA, ca channels) and inB
// (dB, cb channels); accumulate into existing values when acc* != 0.
cudaError_t conv3_dgrad(const ConvDesc& d, const float* dout, float* dA, int accA, float* dB, int accB,
                        cudaStream_t s);
// dW[k][ci][co] += sum_v in[s v + off_k][ci] dOut[v][co],  db[co] += sum_v dOut[v][co]
cudaError_t conv3_wgrad(const ConvDesc& d, const float* dout, float* dw, float* db, cudaStream_t s);

// dy *= leaky'(y) (derivative from the sign of the stored output y)
cudaError_t act_backward(long long n, const __nv_bfloat16* y, float* dy, cudaStream_t s);

// out = P(in) + skip: vertex-centred trilinear prolongation from coarse dims c
// to fine dims f = 2c - 1 (ch channels), plus an optional fine skip tensor.
cudaError_t upsample_forward(const int* cdims, const int* fdims, int ch, const __nv_bfloat16* in,
                             const __nv_bfloat16* skip, __nv_bfloat16* out, const int* skipflag, cudaStream_t s);
// transpose of upsample_forward: coarse gradient += R(fine gradient)
cudaError_t upsample_backward(const int* cdims, const int* fdims, int ch, const float* dfine, float* dcoarse,
                              cudaStream_t s);

// dst += src (FP32)
cudaError_t add_f32(long long n, const float* src, float* dst, cudaStream_t s);

// Network input x[v] = bf16(r[p(v)] * c), v over the nv grid voxels, p(v) =
// p_of_vox[v] (identity when null).  c = sqrt(nv / rr[0]) when rr is given
// (unit-RMS scaling by the residual's squared norm; 0 if rr[0] <= 0), else
// c = scale.  skipflag as in ConvDesc.
cudaError_t unet_input(int nv, const double* r, const int* p_of_vox, const double* rr, double scale,
                       __nv_bfloat16* x, const int* skipflag, cudaStream_t s);
cudaError_t unet_input(int nv, const float* r, const int* p_of_vox, const double* rr, double scale,
                       __nv_bfloat16* x, const int* skipflag, cudaStream_t s);
// Training loss of one sample on grid dims, d = out - target:
//   w_l2 mean(d^2) + w_h1 (1/n) sum over axes of (d[i+e] - d[i])^2
// (neighbour pairs inside the grid); dout = its gradient, lossv[0] += loss.
cudaError_t unet_loss(const int* dims, const float* out, const float* target, float* dout, float* lossv, float w_l2,
                      float w_h1, cudaStream_t s);

// Adam step on FP32 master weights, refreshing the BF16 copy.
cudaError_t adam_step(long long n, float* w, const float* g, float* m, float* v, __nv_bfloat16* wb, float lr,
                      float b1, float b2, float eps, int t, float gscale, cudaStream_t s);

cudaError_t f32_to_bf16(long long n, const float* a, __nv_bfloat16* b, cudaStream_t s);

// ---- tensor-core path (unet_tc.cu): stride-1 and stride-2 convolutions,
// cin in {16, 32, 64}, cout in {16, 32, 64} ----
struct ConvTcParams {
  // TMA descriptor of the input (channels-last BF16, dims cin, x, y, z):
  // box of 8 channels x the halo brick, traversal stride 1 (stride-1
  // layers) or 2 along x, y, z (one parity phase of a stride-2 layer)
  CUtensorMap tmap;
  int dims[3];      // output grid
  int in_dims[3];   // input grid (stride 2: 2 dims - 1 per axis)
  const __nv_bfloat16* in;  // input tensor, channels-last, cin channels
  int stride;       // 1 or 2
  int brick[3];     // output voxels per CTA along each axis
  int nb[3];        // bricks per axis
  int halo[3];      // brick + 2
  int rows;         // rows reserved per 8-channel plane (halo box plus read slack)
  int plane_bytes;  // rows * 16 rounded up to 1 KiB
  int q0, tiles;    // first computed row, 128-row M tiles
  int cin, N, nslices, cout;
  const __nv_bfloat16* wpack;  // conv_tc_pack layout
  const float* bias;
  __nv_bfloat16* out;
  float* out_f32;
  int act;
  const int* skip;
  int* err;  // set when a bounded wait gives up
  // persistent form: shared-memory stages of the halo brick (1 or 2), TMEM
  // columns allocated per CTA and accumulators in the ring; fold = 1: the
  // three dx taps share one MMA (N = 3 nout columns, dx-major), nout output
  // channels per slice
  int astages, acc_cols, nacc, fold, nout;
};
struct ConvTcPlan {
  ConvTcParams p;
  int grid_x;
  size_t smem;
  int ready;
  int pipe;  // 1: the persistent, pipelined kernel (grid_x CTAs, one dimension)
};
bool conv_tc_supported(const ConvDesc& d);
int conv_tc_slice_width(int cin, int cout, int stride);
long long conv_tc_pack_elems(int cin, int cout, int stride);
// Rearranges [27][cin][cout] BF16 weights into per-tap canonical tensor-core
// blocks (wpack holds conv_tc_pack_elems values).
// fold = 1 packs the dx-folded layout of the persistent kernel (stride 1):
// per slice, 9 (dy, dz) groups of N = 3 x slice-width columns, column
// (dx + 1) x width + output channel.  The same number of values.
cudaError_t conv_tc_pack(const __nv_bfloat16* w, int cin, int cout, int stride, __nv_bfloat16* wpack,
                         cudaStream_t s, int fold = 0);
// Builds the launch plan (bricks, shared-memory layout) of a supported
// convolution; 0 on success.  pipe = 1 plans the persistent, pipelined
// kernel instead of one CTA per brick, pipe = 2 that kernel with the dx
// taps folded into N (stride 1 only; the weights packed with fold = 1).
int conv_tc_plan(const ConvDesc& d, const __nv_bfloat16* wpack, int num_sms, ConvTcPlan& plan, int pipe = 0);
// Launches a planned convolution; out_f32 (FP32-output layers) and skip
// replace the plan's pointers for this launch.
cudaError_t conv3_forward_tc(const ConvTcPlan& plan, float* out_f32, const int* skip, int* err, cudaStream_t s);

}  // namespace cfd
