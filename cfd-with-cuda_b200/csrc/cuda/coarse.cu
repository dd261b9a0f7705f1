// Device side of the two-level pressure preconditioners (the coarse space is
// built by galerkin.cu and dense_chol.cu, or on the host by coarse.cpp):
// restriction c = P^T r onto the coarse
// lattice, the coarse solve e = Zc^-1 c as a dense matrix-vector product,
// and the combined preconditioner
//
//   z[p(v)] = D^-1 r[p(v)] + (P e)[v] + s/d * y[v]
//
// (Jacobi step, coarse correction, optional network correction y scaled by
// the residual's RMS s = sqrt(rr / n) and the median diagonal d).  Every
// kernel returns at once while the solve's done flag is set, so the sequence
// can sit inside a captured flexible-CG iteration.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace cfd {

namespace {

// c = P^T r: one warp per coarse node.  The lanes stride over the node's
// support box (at most (2h + 1)^3 fine nodes, x fastest), each adding
// w(x) w(y) w(z) r in FP64 in a fixed order, then a warp sum.  4913 warps
// at 65^3 are resident at once, so the launch is a single wave.
constexpr int kRestrictThreads = 256;
template <class VT>
__global__ void __launch_bounds__(kRestrictThreads) k_restrict(CoarseArgs<VT> a, const VT* __restrict__ r,
                                                               float* __restrict__ c, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  const int node = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (node >= a.nc) return;
  const int cx = a.cd[0], cy = a.cd[1];
  const int ix = node % cx, iy = (node / cx) % cy, iz = node / (cx * cy);
  const int x0 = a.rx[2 * ix], nx = a.rx[2 * ix + 1] - x0 + 1;
  const int y0 = a.ry[2 * iy], ny = a.ry[2 * iy + 1] - y0 + 1;
  const int z0 = a.rz[2 * iz], nz = a.rz[2 * iz + 1] - z0 + 1;
  const int nxy = nx * ny, S = nxy * nz;
  const int fx = a.fd[0], fxy = a.fd[0] * a.fd[1];
  double acc = 0.0;
#pragma unroll 4
  for (int t = lane; t < S; t += 32) {
    const int z = z0 + t / nxy, rem = t - (t / nxy) * nxy;
    const int y = y0 + rem / nx, x = x0 + rem - (rem / nx) * nx;
    const double wx = a.i0x[x] == ix ? 1.0 - a.fx[x] : (a.i0x[x] + 1 == ix ? a.fx[x] : 0.0);
    const double wy = a.i0y[y] == iy ? 1.0 - a.fy[y] : (a.i0y[y] + 1 == iy ? a.fy[y] : 0.0);
    const double wz = a.i0z[z] == iz ? 1.0 - a.fz[z] : (a.i0z[z] + 1 == iz ? a.fz[z] : 0.0);
    const int v = x + fx * y + fxy * z;
    acc += (wx * wy * wz) * (double)r[a.pmap ? a.pmap[v] : v];
  }
  acc = warp_sum(acc);
  if (lane == 0) c[node] = (float)acc;
}

// sum_i h[i] c[i] over 8 FP16 entries packed in q and 8 FP32 values at c
__device__ __forceinline__ float dot8(const uint4& q, const float* c) {
  const __half2* h = reinterpret_cast<const __half2*>(&q);
  const float4 c0 = __ldg(reinterpret_cast<const float4*>(c)), c1 = __ldg(reinterpret_cast<const float4*>(c) + 1);
  float2 f0 = __half22float2(h[0]), f1 = __half22float2(h[1]), f2 = __half22float2(h[2]), f3 = __half22float2(h[3]);
  return (f0.x * c0.x + f0.y * c0.y) + (f1.x * c0.z + f1.y * c0.w) + (f2.x * c1.x + f2.y * c1.y) +
         (f3.x * c1.z + f3.y * c1.w);
}

// e = inv c: one warp per row (eight rows per block), each lane with up to
// eight 16-byte loads (8 FP16 entries each) in flight, FP32 products with c
// (read through L1), warp sum.  All rows' warps are resident at once (4913
// at 65^3), so the launch is a single wave.  The inverse is read with an
// evict-last L2 policy (the SpMV's matrix stream is evict-first).
constexpr int kMvThreads = 256;
template <class VT>
__global__ void __launch_bounds__(kMvThreads) k_coarse_mv(int nc, int ld, const __half* __restrict__ inv, float rscale,
                                                          const float* __restrict__ c, VT* __restrict__ e,
                                                          const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  const int row = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= nc) return;
  const int nv8 = nc >> 3, tail = nc & 7;  // whole 8-entry groups inside the row, then a tail
  const uint4* ir = reinterpret_cast<const uint4*>(inv + (size_t)row * ld);
  const unsigned long long keep = l2_evict_last();
  float s[4] = {0.f, 0.f, 0.f, 0.f};
  int k = lane;
  for (; k + 7 * 32 < nv8; k += 8 * 32) {
    uint4 q[8];
#pragma unroll
    for (int u = 0; u < 8; u++) q[u] = ldg_hint(ir + k + u * 32, keep);
#pragma unroll
    for (int u = 0; u < 8; u++) s[u & 3] += dot8(q[u], c + 8 * (k + u * 32));
  }
  for (; k < nv8; k += 32) s[0] += dot8(ldg_hint(ir + k, keep), c + 8 * k);
  if (lane < tail) s[1] += __half2float(inv[(size_t)row * ld + 8 * nv8 + lane]) * c[8 * nv8 + lane];
  const float t = warp_sum((s[0] + s[1]) + (s[2] + s[3]));
  if (lane == 0) e[row] = (VT)(t * rscale);
}

template <class VT>
__global__ void __launch_bounds__(256) k_precond(CoarseArgs<VT> a, int nv, const VT* __restrict__ r,
                                                 const VT* __restrict__ dinv, const VT* __restrict__ e,
                                                 const float* __restrict__ y, const double* rr, double dscale,
                                                 VT* __restrict__ z, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  VT ys = 0;
  if (y) ys = (VT)(rr[0] > 0.0 ? sqrt(rr[0] / (double)nv) / dscale : 0.0);
  const int cx = a.cd[0], cxy = a.cd[0] * a.cd[1];
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const int p = a.pmap ? a.pmap[v] : v;
    VT zi = dinv[p] * r[p];
    if (e) {
      const int x = v % a.fd[0], yy = (v / a.fd[0]) % a.fd[1], zz = v / (a.fd[0] * a.fd[1]);
      const int ix = a.i0x[x], iy = a.i0y[yy], iz = a.i0z[zz];
      const VT fx = (VT)a.fx[x], fy = (VT)a.fy[yy], fz = (VT)a.fz[zz];
      const int bx = a.cd[0] > 1, by = a.cd[1] > 1, bz = a.cd[2] > 1;
      const VT* e0 = e + ix + cx * iy + cxy * iz;
      VT s = 0;
#pragma unroll
      for (int cnr = 0; cnr < 8; cnr++) {
        const int dx = cnr & 1, dy = (cnr >> 1) & 1, dz = cnr >> 2;
        if ((dx && !bx) || (dy && !by) || (dz && !bz)) continue;
        const VT w = (dx ? fx : 1 - fx) * (dy ? fy : 1 - fy) * (dz ? fz : 1 - fz);
        s += w * e0[dx + cx * dy + cxy * dz];
      }
      zi += s;
    }
    if (y) zi += (VT)y[v] * ys;
    z[p] = zi;
  }
}

int grid_of(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace

template <class VT>
cudaError_t launch_coarse_restrict(const CoarseArgs<VT>& a, const VT* r, float* c, const int* done, cudaStream_t s) {
  const int warps = kRestrictThreads / 32;
  return launch_k(a.pdl != 0, k_restrict<VT>, dim3((a.nc + warps - 1) / warps), dim3(kRestrictThreads), 0, s, a, r,
                  c, done);
}

template <class VT>
cudaError_t launch_coarse_solve(const CoarseArgs<VT>& a, const float* c, VT* e, const int* done, cudaStream_t s) {
  if (a.ldinv % 8 || a.ldinv < a.nc) return cudaErrorInvalidValue;
  const int warps = kMvThreads / 32;
  return launch_k(a.pdl != 0, k_coarse_mv<VT>, dim3((a.nc + warps - 1) / warps), dim3(kMvThreads), 0, s, a.nc,
                  a.ldinv, a.inv16, (float)(1.0 / a.inv_scale), c, e, done);
}

template <class VT>
cudaError_t launch_precond(const CoarseArgs<VT>& a, int nv, const VT* r, const VT* dinv, const VT* e, const float* y,
                           const double* rr, double dscale, VT* z, const int* done, cudaStream_t s) {
  return launch_k(a.pdl != 0, k_precond<VT>, dim3(grid_of(nv, 256)), dim3(256), 0, s, a, nv, r, dinv, e, y, rr,
                  dscale, z, done);
}

template cudaError_t launch_coarse_restrict<float>(const CoarseArgs<float>&, const float*, float*, const int*,
                                                   cudaStream_t);
template cudaError_t launch_coarse_restrict<double>(const CoarseArgs<double>&, const double*, float*, const int*,
                                                    cudaStream_t);
template cudaError_t launch_coarse_solve<float>(const CoarseArgs<float>&, const float*, float*, const int*,
                                                cudaStream_t);
template cudaError_t launch_coarse_solve<double>(const CoarseArgs<double>&, const float*, double*, const int*,
                                                 cudaStream_t);
template cudaError_t launch_precond<float>(const CoarseArgs<float>&, int, const float*, const float*, const float*,
                                           const float*, const double*, double, float*, const int*, cudaStream_t);
template cudaError_t launch_precond<double>(const CoarseArgs<double>&, int, const double*, const double*,
                                            const double*, const float*, const double*, double, double*, const int*,
                                            cudaStream_t);

}  // namespace cfd
