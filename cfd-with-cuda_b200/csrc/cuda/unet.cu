// U-Net preconditioner kernels: 3x3x3 convolutions (stride 1 or 2) on
// channels-last BF16 activations with BF16 weights and FP32 accumulation,
// their data- and weight-gradients, vertex-centred prolongation and its
// transpose, input scaling, MSE loss and Adam.  These are the training and
// reference kernels; the inference hot path uses the tensor-core forward
// convolution in unet_tc.cu where the layer shape allows.
#include <cuda_bf16.h>

#include "common.cuh"
#include "unet.h"

namespace cfd {

namespace {

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

struct Dims3 {
  int c[3], f[3];  // coarse and fine grid dims
};

__device__ __forceinline__ void vox3(long long v, const int* d, int& x, int& y, int& z) {
  x = (int)(v % d[0]);
  long long t = v / d[0];
  y = (int)(t % d[1]);
  z = (int)(t / d[1]);
}

// One thread per output voxel, COB output channels per block row (blockIdx.y
// = output-channel chunk); the weight chunk [27][cin][COB] is staged in
// shared memory as FP32 and read as warp-wide broadcasts.
template <int COB>
__global__ void __launch_bounds__(128) k_conv_fwd(ConvDesc d) {
  extern __shared__ float sw[];
  if (d.skip && *d.skip) return;
  const int cin = d.ca + d.cb, co0 = blockIdx.y * COB;
  for (int i = threadIdx.x; i < 27 * cin * COB; i += blockDim.x) {
    const int co = i % COB, ci = (i / COB) % cin, k = i / (COB * cin);
    sw[i] = (co0 + co < d.cout) ? bf(d.w[((size_t)k * cin + ci) * d.cout + co0 + co]) : 0.f;
  }
  __syncthreads();
  const long long nv = (long long)d.out_dims[0] * d.out_dims[1] * d.out_dims[2];
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv;
       v += (long long)gridDim.x * blockDim.x) {
    int X, Y, Z;
    vox3(v, d.out_dims, X, Y, Z);
    float acc[COB];
#pragma unroll
    for (int c = 0; c < COB; c++) acc[c] = (co0 + c < d.cout) ? d.bias[co0 + c] : 0.f;
    for (int k = 0; k < 27; k++) {
      const int ix = X * d.stride + (k % 3) - 1, iy = Y * d.stride + (k / 3) % 3 - 1, iz = Z * d.stride + k / 9 - 1;
      if (ix < 0 || iy < 0 || iz < 0 || ix >= d.in_dims[0] || iy >= d.in_dims[1] || iz >= d.in_dims[2]) continue;
      const long long u = ix + (long long)d.in_dims[0] * (iy + (long long)d.in_dims[1] * iz);
      const float* wk = sw + (size_t)k * cin * COB;
      const __nv_bfloat16* a = d.inA + u * d.ca;
      for (int ci = 0; ci < d.ca; ci++) {
        const float x = bf(a[ci]);
#pragma unroll
        for (int c = 0; c < COB; c++) acc[c] += x * wk[ci * COB + c];
      }
      if (d.cb) {
        const __nv_bfloat16* b = d.inB + u * d.cb;
        wk += (size_t)d.ca * COB;
        for (int ci = 0; ci < d.cb; ci++) {
          const float x = bf(b[ci]);
#pragma unroll
          for (int c = 0; c < COB; c++) acc[c] += x * wk[ci * COB + c];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < COB; c++) {
      if (co0 + c >= d.cout) break;
      float y = acc[c];
      if (d.act && y < 0.f) y *= kLeaky;
      if (d.out) d.out[v * d.cout + co0 + c] = __float2bfloat16(y);
      if (d.out_f32) d.out_f32[v * d.cout + co0 + c] = y;
    }
  }
}

// Sixteen-input-channel convolution with a single FP32 output (the last
// layer).  A block computes a 16 x 4 x 4 tile of output voxels, one per
// thread: the tile's inputs plus a one-voxel halo (18 x 6 x 6 voxels of 16
// BF16 channels, zero outside the grid) are loaded into shared memory once
// with 16-byte loads, so each input voxel comes from L2 about 2.5 times
// instead of 27; the 27 x 16 weights sit in shared memory as float4 rows.
// The taps are summed in the same order as a direct loop over them.
constexpr int k16X = 16, k16Y = 4, k16Z = 4;
__global__ void __launch_bounds__(k16X * k16Y * k16Z) k_conv_16to1(ConvDesc d) {
  constexpr int HX = k16X + 2, HY = k16Y + 2, HZ = k16Z + 2;
  __shared__ uint4 tile[HX * HY * HZ][2];
  __shared__ float4 sw[27 * 4];
  if (d.skip && *d.skip) return;
  for (int i = threadIdx.x; i < 27 * 16; i += blockDim.x) ((float*)sw)[i] = bf(d.w[i]);
  const float b0 = d.bias[0];
  const int nx = d.out_dims[0], ny = d.out_dims[1], nz = d.out_dims[2];
  const int tbx = (nx + k16X - 1) / k16X, tby = (ny + k16Y - 1) / k16Y;
  const int bx = blockIdx.x % tbx, by = (blockIdx.x / tbx) % tby, bz = blockIdx.x / (tbx * tby);
  const int x0 = bx * k16X, y0 = by * k16Y, z0 = bz * k16Z;
  for (int i = threadIdx.x; i < HX * HY * HZ * 2; i += blockDim.x) {
    const int vox = i >> 1, half = i & 1;
    const int hx = vox % HX, hy = (vox / HX) % HY, hz = vox / (HX * HY);
    const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
    uint4 u = make_uint4(0, 0, 0, 0);
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < nx && gy < ny && gz < nz)
      u = __ldg(reinterpret_cast<const uint4*>(d.inA + ((size_t)gx + (size_t)nx * (gy + (size_t)ny * gz)) * 16) +
                half);
    tile[vox][half] = u;
  }
  __syncthreads();
  const int tx = threadIdx.x % k16X, ty = (threadIdx.x / k16X) % k16Y, tz = threadIdx.x / (k16X * k16Y);
  const int x = x0 + tx, y = y0 + ty, z = z0 + tz;
  if (x >= nx || y >= ny || z >= nz) return;
  float acc = b0;
#pragma unroll 3
  for (int k = 0; k < 27; k++) {
    const int vox = (tx + k % 3) + HX * ((ty + (k / 3) % 3) + HY * (tz + k / 9));
    const uint4 u0 = tile[vox][0], u1 = tile[vox][1];
    const __nv_bfloat162* h0 = reinterpret_cast<const __nv_bfloat162*>(&u0);
    const __nv_bfloat162* h1 = reinterpret_cast<const __nv_bfloat162*>(&u1);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float4 w = sw[4 * k + q];
      const float2 a = __bfloat1622float2(q < 2 ? h0[2 * q] : h1[2 * (q - 2)]);
      const float2 b = __bfloat1622float2(q < 2 ? h0[2 * q + 1] : h1[2 * (q - 2) + 1]);
      acc += a.x * w.x + a.y * w.y + b.x * w.z + b.y * w.w;
    }
  }
  if (d.act && acc < 0.f) acc *= kLeaky;
  d.out_f32[(size_t)x + (size_t)nx * (y + (size_t)ny * z)] = acc;
}

// Single-input-channel convolution (the first layer) with 16 outputs.  A
// block computes a 16 x 4 x 4 tile of output voxels, one per thread: the
// tile's input plus a one-voxel halo (18 x 6 x 6 values, zero outside the
// grid) is staged in shared memory as FP32, the 27 x 16 weights as float4
// rows (each read is a broadcast), and a thread keeps its 16 sums in
// registers.  The taps are summed in order 0..26 per channel, starting from
// the bias, as a direct loop over them.
__global__ void __launch_bounds__(k16X * k16Y * k16Z) k_conv_c1to16(ConvDesc d) {
  constexpr int HX = k16X + 2, HY = k16Y + 2, HZ = k16Z + 2;
  __shared__ float tile[HX * HY * HZ];
  __shared__ float4 sw[27 * 4];
  __shared__ float sb[16];
  if (d.skip && *d.skip) return;
  for (int i = threadIdx.x; i < 27 * 16; i += blockDim.x) ((float*)sw)[i] = bf(d.w[i]);
  if (threadIdx.x < 16) sb[threadIdx.x] = d.bias[threadIdx.x];
  const int nx = d.out_dims[0], ny = d.out_dims[1], nz = d.out_dims[2];
  const int tbx = (nx + k16X - 1) / k16X, tby = (ny + k16Y - 1) / k16Y;
  const int bx = blockIdx.x % tbx, by = (blockIdx.x / tbx) % tby, bz = blockIdx.x / (tbx * tby);
  const int x0 = bx * k16X, y0 = by * k16Y, z0 = bz * k16Z;
  for (int i = threadIdx.x; i < HX * HY * HZ; i += blockDim.x) {
    const int hx = i % HX, hy = (i / HX) % HY, hz = i / (HX * HY);
    const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
    float u = 0.f;
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < nx && gy < ny && gz < nz)
      u = bf(d.inA[(size_t)gx + (size_t)nx * (gy + (size_t)ny * gz)]);
    tile[i] = u;
  }
  __syncthreads();
  const int tx = threadIdx.x % k16X, ty = (threadIdx.x / k16X) % k16Y, tz = threadIdx.x / (k16X * k16Y);
  const int x = x0 + tx, y = y0 + ty, z = z0 + tz;
  if (x >= nx || y >= ny || z >= nz) return;
  float acc[16];
#pragma unroll
  for (int c = 0; c < 16; c++) acc[c] = sb[c];
#pragma unroll 3
  for (int k = 0; k < 27; k++) {
    const float a = tile[(tx + k % 3) + HX * ((ty + (k / 3) % 3) + HY * (tz + k / 9))];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float4 w = sw[4 * k + q];
      acc[4 * q] += a * w.x;
      acc[4 * q + 1] += a * w.y;
      acc[4 * q + 2] += a * w.z;
      acc[4 * q + 3] += a * w.w;
    }
  }
  __align__(16) __nv_bfloat16 o[16];
#pragma unroll
  for (int c = 0; c < 16; c++) {
    float yv = acc[c];
    if (d.act && yv < 0.f) yv *= kLeaky;
    o[c] = __float2bfloat16(yv);
  }
  const size_t v = (size_t)x + (size_t)nx * (y + (size_t)ny * z);
  uint4* dst = (uint4*)(d.out + v * 16);
  dst[0] = ((const uint4*)o)[0];
  dst[1] = ((const uint4*)o)[1];
}

// Prolongation plus skip for CH channels: one thread per fine voxel, 16-byte
// vector loads and stores, 32-bit index arithmetic.  The corners are summed
// in the order (z, y, x) of the coarse cell, as the trilinear weights of the
// fine index pick them.
template <int CH>
__global__ void __launch_bounds__(256) k_up_fwd_v(Dims3 g, const __nv_bfloat16* __restrict__ in,
                                                  const __nv_bfloat16* __restrict__ skip, __nv_bfloat16* out,
                                                  const int* skipflag) {
  if (skipflag && *skipflag) return;
  const int fx = g.f[0], fy = g.f[1], fz = g.f[2], cx = g.c[0], cy = g.c[1];
  const int nf = fx * fy * fz;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nf; v += gridDim.x * blockDim.x) {
    const int X = v % fx, t = v / fx, Y = t % fy, Z = t / fy;
    float acc[CH];
#pragma unroll
    for (int c = 0; c < CH; c++) acc[c] = 0.f;
    const float w = ((X & 1) ? 0.5f : 1.f) * ((Y & 1) ? 0.5f : 1.f) * ((Z & 1) ? 0.5f : 1.f);
    // the (up to) 8 coarse corners, all loads issued before any sum; a
    // corner an even fine index does not use is read at a clamped index and
    // adds zero
    uint4 u[8][CH / 8];
#pragma unroll
    for (int cnr = 0; cnr < 8; cnr++) {
      const int xx = cnr & 1, yy = (cnr >> 1) & 1, zz = cnr >> 2;
      const int ix = min((X >> 1) + xx, cx - 1), iy = min((Y >> 1) + yy, cy - 1);
      const int iz = min((Z >> 1) + zz, g.c[2] - 1);
      const uint4* src = (const uint4*)(in + (size_t)(ix + cx * (iy + cy * iz)) * CH);
#pragma unroll
      for (int q = 0; q < CH / 8; q++) u[cnr][q] = src[q];
    }
#pragma unroll
    for (int cnr = 0; cnr < 8; cnr++) {
      const int xx = cnr & 1, yy = (cnr >> 1) & 1, zz = cnr >> 2;
      const bool used = (!xx || (X & 1)) && (!yy || (Y & 1)) && (!zz || (Z & 1));
#pragma unroll
      for (int q = 0; q < CH / 8; q++) {
        const __nv_bfloat16* h = (const __nv_bfloat16*)&u[cnr][q];
#pragma unroll
        for (int i = 0; i < 8; i++) acc[8 * q + i] += used ? bf(h[i]) : 0.f;
      }
    }
    const uint4* sk = (const uint4*)(skip + (size_t)v * CH);
    uint4* dst = (uint4*)(out + (size_t)v * CH);
#pragma unroll
    for (int q = 0; q < CH / 8; q++) {
      uint4 u = sk[q];
      const __nv_bfloat16* h = (const __nv_bfloat16*)&u;
      __align__(16) __nv_bfloat16 o[8];
#pragma unroll
      for (int i = 0; i < 8; i++) o[i] = __float2bfloat16(acc[8 * q + i] * w + bf(h[i]));
      dst[q] = *(const uint4*)o;
    }
  }
}

// One thread per input voxel, CIB input channels per blockIdx.y chunk;
// weights staged as [27][cout][CIB].
template <int CIB>
__global__ void __launch_bounds__(128) k_conv_dgrad(ConvDesc d, const float* __restrict__ dout, float* dA, int accA,
                                                    float* dB, int accB) {
  extern __shared__ float sw[];
  const int cin = d.ca + d.cb, ci0 = blockIdx.y * CIB;
  for (int i = threadIdx.x; i < 27 * d.cout * CIB; i += blockDim.x) {
    const int c = i % CIB, co = (i / CIB) % d.cout, k = i / (CIB * d.cout);
    sw[i] = (ci0 + c < cin) ? bf(d.w[((size_t)k * cin + ci0 + c) * d.cout + co]) : 0.f;
  }
  __syncthreads();
  const long long nu = (long long)d.in_dims[0] * d.in_dims[1] * d.in_dims[2];
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < nu;
       u += (long long)gridDim.x * blockDim.x) {
    int ix, iy, iz;
    vox3(u, d.in_dims, ix, iy, iz);
    float acc[CIB];
#pragma unroll
    for (int c = 0; c < CIB; c++) acc[c] = 0.f;
    for (int k = 0; k < 27; k++) {
      int X = ix - ((k % 3) - 1), Y = iy - ((k / 3) % 3 - 1), Z = iz - (k / 9 - 1);
      if (d.stride == 2) {
        if ((X | Y | Z) & 1) continue;
        X >>= 1;
        Y >>= 1;
        Z >>= 1;
      }
      if (X < 0 || Y < 0 || Z < 0 || X >= d.out_dims[0] || Y >= d.out_dims[1] || Z >= d.out_dims[2]) continue;
      const long long v = X + (long long)d.out_dims[0] * (Y + (long long)d.out_dims[1] * Z);
      const float* g = dout + v * d.cout;
      const float* wk = sw + (size_t)k * d.cout * CIB;
      for (int co = 0; co < d.cout; co++) {
        const float gv = g[co];
#pragma unroll
        for (int c = 0; c < CIB; c++) acc[c] += gv * wk[co * CIB + c];
      }
    }
#pragma unroll
    for (int c = 0; c < CIB; c++) {
      const int ci = ci0 + c;
      if (ci >= cin) break;
      if (ci < d.ca) {
        if (dA) {
          float* p = dA + u * d.ca + ci;
          *p = accA ? *p + acc[c] : acc[c];
        }
      } else if (dB) {
        float* p = dB + u * d.cb + (ci - d.ca);
        *p = accB ? *p + acc[c] : acc[c];
      }
    }
  }
}

// Weight gradient: blockIdx.x = voxel chunk, blockIdx.y = tap k, blockIdx.z =
// input-channel chunk of CIB; a tile of TV output voxels of the input values
// and output gradients is staged in shared memory; thread t accumulates the
// (ci, co) pairs t, t + blockDim, ...; partial sums are added atomically.
constexpr int kTV = 32;
constexpr int kWgJ = 2;  // (ci, co) pairs per thread: CIB * cout <= kWgJ * 256
template <int CIB>
__global__ void __launch_bounds__(256) k_conv_wgrad(ConvDesc d, const float* __restrict__ dout, float* dw,
                                                    long long vchunk) {
  __shared__ float s_in[kTV][CIB];
  extern __shared__ float s_g[];  // [kTV][cout]
  const int cin = d.ca + d.cb, k = blockIdx.y, ci0 = blockIdx.z * CIB;
  const long long nv = (long long)d.out_dims[0] * d.out_dims[1] * d.out_dims[2];
  const long long v0 = blockIdx.x * vchunk, v1 = v0 + vchunk < nv ? v0 + vchunk : nv;
  const int npair = CIB * d.cout;
  float acc[kWgJ];
#pragma unroll
  for (int j = 0; j < kWgJ; j++) acc[j] = 0.f;
  const int dx = (k % 3) - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
  for (long long t0 = v0; t0 < v1; t0 += kTV) {
    __syncthreads();
    for (int i = threadIdx.x; i < kTV * CIB; i += blockDim.x) {
      const int tv = i / CIB, c = i % CIB;
      const long long v = t0 + tv;
      float val = 0.f;
      if (v < v1 && ci0 + c < cin) {
        int X, Y, Z;
        vox3(v, d.out_dims, X, Y, Z);
        const int ix = X * d.stride + dx, iy = Y * d.stride + dy, iz = Z * d.stride + dz;
        if (ix >= 0 && iy >= 0 && iz >= 0 && ix < d.in_dims[0] && iy < d.in_dims[1] && iz < d.in_dims[2]) {
          const long long u = ix + (long long)d.in_dims[0] * (iy + (long long)d.in_dims[1] * iz);
          const int ci = ci0 + c;
          val = ci < d.ca ? bf(d.inA[u * d.ca + ci]) : bf(d.inB[u * d.cb + (ci - d.ca)]);
        }
      }
      s_in[tv][c] = val;
    }
    for (int i = threadIdx.x; i < kTV * d.cout; i += blockDim.x) {
      const int tv = i / d.cout, co = i % d.cout;
      const long long v = t0 + tv;
      s_g[i] = v < v1 ? dout[v * d.cout + co] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kWgJ; j++) {
      const int pr = threadIdx.x + j * blockDim.x;
      if (pr < npair) {
        const int c = pr / d.cout, co = pr % d.cout;
        float a = 0.f;
#pragma unroll 8
        for (int tv = 0; tv < kTV; tv++) a += s_in[tv][c] * s_g[tv * d.cout + co];
        acc[j] += a;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kWgJ; j++) {
    const int pr = threadIdx.x + j * blockDim.x;
    if (pr < npair) {
      const int c = pr / d.cout, co = pr % d.cout;
      if (ci0 + c < cin) atomicAdd(dw + ((size_t)k * cin + ci0 + c) * d.cout + co, acc[j]);
    }
  }
}

__global__ void k_bias_grad(long long nv, int cout, const float* __restrict__ dout, float* db, long long vchunk) {
  const long long v0 = blockIdx.x * vchunk, v1 = v0 + vchunk < nv ? v0 + vchunk : nv;
  for (int co = threadIdx.x; co < cout; co += blockDim.x) {
    float a = 0.f;
    for (long long v = v0; v < v1; v++) a += dout[v * cout + co];
    atomicAdd(db + co, a);
  }
}

__global__ void k_act_bwd(long long n, const __nv_bfloat16* __restrict__ y, float* dy) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (bf(y[i]) <= 0.f) dy[i] *= kLeaky;
}


__global__ void k_up_fwd(Dims3 g, int ch, const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* skip,
                         __nv_bfloat16* out, const int* skipflag) {
  if (skipflag && *skipflag) return;
  const long long nf = (long long)g.f[0] * g.f[1] * g.f[2];
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nf * ch;
       v += (long long)gridDim.x * blockDim.x) {
    const long long fv = v / ch;
    const int c = (int)(v % ch);
    int X, Y, Z;
    vox3(fv, g.f, X, Y, Z);
    const int x0 = X >> 1, x1 = (X + 1) >> 1, y0 = Y >> 1, y1 = (Y + 1) >> 1, z0 = Z >> 1, z1 = (Z + 1) >> 1;
    const float wx = (X & 1) ? 0.5f : 1.f, wy = (Y & 1) ? 0.5f : 1.f, wz = (Z & 1) ? 0.5f : 1.f;
    float s = 0.f;
    for (int zz = 0; zz < ((Z & 1) ? 2 : 1); zz++)
      for (int yy = 0; yy < ((Y & 1) ? 2 : 1); yy++)
        for (int xx = 0; xx < ((X & 1) ? 2 : 1); xx++) {
          const int cx = xx ? x1 : x0, cy = yy ? y1 : y0, cz = zz ? z1 : z0;
          s += bf(in[((long long)cx + (long long)g.c[0] * (cy + (long long)g.c[1] * cz)) * ch + c]);
        }
    s *= wx * wy * wz;
    if (skip) s += bf(skip[v]);
    out[v] = __float2bfloat16(s);
  }
}

__global__ void k_up_bwd(Dims3 g, int ch, const float* __restrict__ dfine, float* dcoarse) {
  const long long nc = (long long)g.c[0] * g.c[1] * g.c[2];
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nc * ch;
       v += (long long)gridDim.x * blockDim.x) {
    const long long cv = v / ch;
    const int c = (int)(v % ch);
    int x, y, z;
    vox3(cv, g.c, x, y, z);
    float s = 0.f;
    for (int dz = -1; dz <= 1; dz++) {
      const int Z = 2 * z + dz;
      if (Z < 0 || Z >= g.f[2]) continue;
      const float wz = dz ? 0.5f : 1.f;
      for (int dy = -1; dy <= 1; dy++) {
        const int Y = 2 * y + dy;
        if (Y < 0 || Y >= g.f[1]) continue;
        const float wy = dy ? 0.5f : 1.f;
        for (int dx = -1; dx <= 1; dx++) {
          const int X = 2 * x + dx;
          if (X < 0 || X >= g.f[0]) continue;
          const float wx = dx ? 0.5f : 1.f;
          s += wx * wy * wz * dfine[((long long)X + (long long)g.f[0] * (Y + (long long)g.f[1] * Z)) * ch + c];
        }
      }
    }
    dcoarse[v] += s;
  }
}

template <class T>
__global__ void k_input(int nv, const T* __restrict__ r, const int* __restrict__ pmap, const double* rr,
                        double scale, __nv_bfloat16* x, const int* skipflag) {
  if (skipflag && *skipflag) return;
  double c = scale;
  if (rr) c = rr[0] > 0.0 ? sqrt((double)nv / rr[0]) : 0.0;
  const float cf = (float)c;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
    x[i] = __float2bfloat16((float)r[pmap ? pmap[i] : i] * cf);
}
__global__ void k_add(long long n, const float* __restrict__ a, float* b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] += a[i];
}

__global__ void k_loss(Dims3 g, const float* __restrict__ out, const float* __restrict__ t, float* dout,
                       float* lossv, float wl2, float wh1) {
  const int nx = g.f[0], ny = g.f[1], nz = g.f[2];
  const long long n = (long long)nx * ny * nz;
  const float inv = 1.f / (float)n;
  double v[1] = {0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    vox3(i, g.f, x, y, z);
    const float di = out[i] - t[i];
    float gi = 2.f * wl2 * di;
    double li = (double)wl2 * di * di;
    if (wh1 != 0.f) {
      const long long st[3] = {1, nx, (long long)nx * ny};
      const int c[3] = {x, y, z}, m[3] = {nx, ny, nz};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        if (c[a] + 1 < m[a]) {
          const float dn = out[i + st[a]] - t[i + st[a]];
          gi += 2.f * wh1 * (di - dn);
          li += (double)wh1 * (dn - di) * (dn - di);
        }
        if (c[a] > 0) gi += 2.f * wh1 * (di - (out[i - st[a]] - t[i - st[a]]));
      }
    }
    dout[i] = gi * inv;
    v[0] += li;
  }
  block_sum<1>(v);
  if (threadIdx.x == 0) atomicAdd(lossv, (float)(v[0] / n));
}

__global__ void k_adam(long long n, float* w, const float* __restrict__ g, float* m, float* v, __nv_bfloat16* wb,
                       float lr, float b1, float b2, float eps, float bc1, float bc2, float gscale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wn = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wn;
    if (wb) wb[i] = __float2bfloat16(wn);
  }
}

__global__ void k_f2bf(long long n, const float* __restrict__ a, __nv_bfloat16* b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16(a[i]);
}

int grid1(long long n, int t = 256) {
  long long g = (n + t - 1) / t;
  if (g > 148 * 32) g = 148 * 32;
  return (int)(g < 1 ? 1 : g);
}

// Raises the kernel's dynamic shared-memory limit to the largest a block may
// have when a launch needs more than the default: the limit belongs to the
// kernel, and launches of other layers (or recorded in a CUDA graph) must
// stay valid.
template <class F>
cudaError_t with_smem(F kernel, size_t bytes) {
  if (bytes > 48 * 1024) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  return cudaSuccess;
}

}  // namespace

cudaError_t conv3_forward(const ConvDesc& d, cudaStream_t s) {
  const int cin = d.ca + d.cb;
  const long long nv = (long long)d.out_dims[0] * d.out_dims[1] * d.out_dims[2];
  const int gx = grid1(nv, 128);
  if (cin == 1 && d.cout == 16 && d.stride == 1 && d.out && !d.out_f32 && nv < (1LL << 31)) {
    const long long tiles = (long long)((d.out_dims[0] + k16X - 1) / k16X) * ((d.out_dims[1] + k16Y - 1) / k16Y) *
                            ((d.out_dims[2] + k16Z - 1) / k16Z);
    k_conv_c1to16<<<(unsigned)tiles, k16X * k16Y * k16Z, 0, s>>>(d);
    return cudaGetLastError();
  }
  if (d.ca == 16 && d.cb == 0 && d.cout == 1 && d.stride == 1 && d.out_f32 && !d.out && nv < (1LL << 31)) {
    const long long tiles = (long long)((d.out_dims[0] + k16X - 1) / k16X) * ((d.out_dims[1] + k16Y - 1) / k16Y) *
                            ((d.out_dims[2] + k16Z - 1) / k16Z);
    k_conv_16to1<<<(unsigned)tiles, k16X * k16Y * k16Z, 0, s>>>(d);
    return cudaGetLastError();
  }
  if (cin <= 48) {
    const size_t sm = (size_t)27 * cin * 16 * sizeof(float);
    cudaError_t e = with_smem(k_conv_fwd<16>, sm);
    if (e != cudaSuccess) return e;
    k_conv_fwd<16><<<dim3(gx, (d.cout + 15) / 16), 128, sm, s>>>(d);
  } else {
    const size_t sm = (size_t)27 * cin * 8 * sizeof(float);
    cudaError_t e = with_smem(k_conv_fwd<8>, sm);
    if (e != cudaSuccess) return e;
    k_conv_fwd<8><<<dim3(gx, (d.cout + 7) / 8), 128, sm, s>>>(d);
  }
  return cudaGetLastError();
}

cudaError_t conv3_dgrad(const ConvDesc& d, const float* dout, float* dA, int accA, float* dB, int accB,
                        cudaStream_t s) {
  const int cin = d.ca + d.cb;
  const long long nu = (long long)d.in_dims[0] * d.in_dims[1] * d.in_dims[2];
  const int gx = grid1(nu, 128);
  if (d.cout <= 32) {
    const size_t sm = (size_t)27 * d.cout * 16 * sizeof(float);
    cudaError_t e = with_smem(k_conv_dgrad<16>, sm);
    if (e != cudaSuccess) return e;
    k_conv_dgrad<16><<<dim3(gx, (cin + 15) / 16), 128, sm, s>>>(d, dout, dA, accA, dB, accB);
  } else {
    const size_t sm = (size_t)27 * d.cout * 8 * sizeof(float);
    cudaError_t e = with_smem(k_conv_dgrad<8>, sm);
    if (e != cudaSuccess) return e;
    k_conv_dgrad<8><<<dim3(gx, (cin + 7) / 8), 128, sm, s>>>(d, dout, dA, accA, dB, accB);
  }
  return cudaGetLastError();
}

cudaError_t conv3_wgrad(const ConvDesc& d, const float* dout, float* dw, float* db, cudaStream_t s) {
  const int cin = d.ca + d.cb;
  const long long nv = (long long)d.out_dims[0] * d.out_dims[1] * d.out_dims[2];
  const long long vchunk = 2048;
  const int nchunk = (int)((nv + vchunk - 1) / vchunk);
  // CIB chosen so that CIB * cout <= kWgJ * 256
  const size_t sm = (size_t)kTV * d.cout * sizeof(float);
  if (d.cout <= 64) {
    if (d.cout <= 32) {
      k_conv_wgrad<16><<<dim3(nchunk, 27, (cin + 15) / 16), 256, sm, s>>>(d, dout, dw, vchunk);
    } else {
      k_conv_wgrad<8><<<dim3(nchunk, 27, (cin + 7) / 8), 256, sm, s>>>(d, dout, dw, vchunk);
    }
  } else {
    return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (db) {
    const long long bchunk = 1024;
    k_bias_grad<<<(int)((nv + bchunk - 1) / bchunk), 64, 0, s>>>(nv, d.cout, dout, db, bchunk);
  }
  return cudaGetLastError();
}

cudaError_t act_backward(long long n, const __nv_bfloat16* y, float* dy, cudaStream_t s) {
  k_act_bwd<<<grid1(n), 256, 0, s>>>(n, y, dy);
  return cudaGetLastError();
}

cudaError_t upsample_forward(const int* cdims, const int* fdims, int ch, const __nv_bfloat16* in,
                             const __nv_bfloat16* skip, __nv_bfloat16* out, const int* skipflag, cudaStream_t s) {
  Dims3 g;
  for (int i = 0; i < 3; i++) {
    g.c[i] = cdims[i];
    g.f[i] = fdims[i];
  }
  const long long nf = (long long)fdims[0] * fdims[1] * fdims[2];
  if (skip && nf < (1LL << 31) && (ch == 16 || ch == 32)) {
    if (ch == 16)
      k_up_fwd_v<16><<<grid1(nf), 256, 0, s>>>(g, in, skip, out, skipflag);
    else
      k_up_fwd_v<32><<<grid1(nf), 256, 0, s>>>(g, in, skip, out, skipflag);
    return cudaGetLastError();
  }
  const long long n = nf * ch;
  k_up_fwd<<<grid1(n), 256, 0, s>>>(g, ch, in, skip, out, skipflag);
  return cudaGetLastError();
}

cudaError_t upsample_backward(const int* cdims, const int* fdims, int ch, const float* dfine, float* dcoarse,
                              cudaStream_t s) {
  Dims3 g;
  for (int i = 0; i < 3; i++) {
    g.c[i] = cdims[i];
    g.f[i] = fdims[i];
  }
  const long long n = (long long)cdims[0] * cdims[1] * cdims[2] * ch;
  k_up_bwd<<<grid1(n), 256, 0, s>>>(g, ch, dfine, dcoarse);
  return cudaGetLastError();
}

cudaError_t add_f32(long long n, const float* src, float* dst, cudaStream_t s) {
  k_add<<<grid1(n), 256, 0, s>>>(n, src, dst);
  return cudaGetLastError();
}

cudaError_t unet_input(int nv, const double* r, const int* pmap, const double* rr, double scale,
                       __nv_bfloat16* x, const int* skipflag, cudaStream_t s) {
  k_input<double><<<grid1(nv), 256, 0, s>>>(nv, r, pmap, rr, scale, x, skipflag);
  return cudaGetLastError();
}
cudaError_t unet_input(int nv, const float* r, const int* pmap, const double* rr, double scale,
                       __nv_bfloat16* x, const int* skipflag, cudaStream_t s) {
  k_input<float><<<grid1(nv), 256, 0, s>>>(nv, r, pmap, rr, scale, x, skipflag);
  return cudaGetLastError();
}
cudaError_t unet_loss(const int* dims, const float* out, const float* target, float* dout, float* lossv, float w_l2,
                      float w_h1, cudaStream_t s) {
  Dims3 g;
  for (int i = 0; i < 3; i++) g.c[i] = g.f[i] = dims[i];
  const long long n = (long long)dims[0] * dims[1] * dims[2];
  k_loss<<<grid1(n), 256, 0, s>>>(g, out, target, dout, lossv, w_l2, w_h1);
  return cudaGetLastError();
}

cudaError_t adam_step(long long n, float* w, const float* g, float* m, float* v, __nv_bfloat16* wb, float lr,
                      float b1, float b2, float eps, int t, float gscale, cudaStream_t s) {
  const float bc1 = 1.f - powf(b1, (float)t), bc2 = 1.f - powf(b2, (float)t);
  k_adam<<<grid1(n), 256, 0, s>>>(n, w, g, m, v, wb, lr, b1, b2, eps, bc1, bc2, gscale);
  return cudaGetLastError();
}

cudaError_t f32_to_bf16(long long n, const float* a, __nv_bfloat16* b, cudaStream_t s) {
  k_f2bf<<<grid1(n), 256, 0, s>>>(n, a, b);
  return cudaGetLastError();
}

}  // namespace cfd
