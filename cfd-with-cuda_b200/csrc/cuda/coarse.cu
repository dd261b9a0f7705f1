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

// c = P^T r, separably: one block per coarse (iy, iz) pair.  The block's
// fine x-lines (the y-z support of the pair, weights wy wz kept in shared
// memory) are summed by G groups of fd[0] threads, each thread one fine x
// over every G-th line (independent loads), the group partials are added,
// and warps restrict the resulting fine x-line onto the coarse x-nodes.
constexpr int kRestrictThreads = 512;
constexpr int kRestrictLines = 1024;  // y-z support lines per coarse pair at most
template <class VT>
__global__ void __launch_bounds__(kRestrictThreads) k_restrict(CoarseArgs<VT> a, const VT* __restrict__ r,
                                                               float* __restrict__ c, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  extern __shared__ double sline[];  // G x fd[0] partial sums
  __shared__ double swt[kRestrictLines];
  __shared__ int sbase[kRestrictLines];
  const int cx = a.cd[0], cy = a.cd[1];
  const int iy = blockIdx.x % cy, iz = blockIdx.x / cy;
  const int y0 = a.ry[2 * iy], ny = a.ry[2 * iy + 1] - y0 + 1;
  const int z0 = a.rz[2 * iz], nz = a.rz[2 * iz + 1] - z0 + 1;
  const int fx = a.fd[0], fxy = a.fd[0] * a.fd[1];
  const int nl = ny * nz;
  for (int l = threadIdx.x; l < nl; l += blockDim.x) {
    const int y = y0 + l % ny, z = z0 + l / ny;
    const double wy = a.i0y[y] == iy ? 1.0 - a.fy[y] : (a.i0y[y] + 1 == iy ? a.fy[y] : 0.0);
    const double wz = a.i0z[z] == iz ? 1.0 - a.fz[z] : (a.i0z[z] + 1 == iz ? a.fz[z] : 0.0);
    swt[l] = wy * wz;
    sbase[l] = fx * y + fxy * z;
  }
  __syncthreads();
  const int G = fx <= (int)blockDim.x ? (int)blockDim.x / fx : 1;
  const int g = threadIdx.x / fx;
  for (int x = threadIdx.x % fx; g < G && x < fx; x += (G == 1 ? (int)blockDim.x : fx)) {
    double acc = 0.0;
#pragma unroll 4
    for (int l = g; l < nl; l += G) {
      const int v = sbase[l] + x;
      acc += swt[l] * (double)r[a.pmap ? a.pmap[v] : v];
    }
    sline[g * fx + x] = acc;
    if (G != 1) break;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int ix = warp; ix < cx; ix += blockDim.x >> 5) {
    const int x0 = a.rx[2 * ix], x1 = a.rx[2 * ix + 1];
    double acc = 0.0;
    for (int x = x0 + lane; x <= x1; x += 32) {
      const double wx = a.i0x[x] == ix ? 1.0 - a.fx[x] : (a.i0x[x] + 1 == ix ? a.fx[x] : 0.0);
      double sx = 0.0;
      for (int gg = 0; gg < G; gg++) sx += sline[gg * fx + x];
      acc += wx * sx;
    }
    acc = warp_sum(acc);
    if (lane == 0) c[ix + cx * (iy + cy * iz)] = (float)acc;
  }
}

// sum_i h[i] c[i] over 8 FP16 entries packed in q and 8 FP32 values at c
__device__ __forceinline__ float dot8(const uint4& q, const float* c) {
  const __half2* h = reinterpret_cast<const __half2*>(&q);
  const float4 c0 = __ldg(reinterpret_cast<const float4*>(c)), c1 = __ldg(reinterpret_cast<const float4*>(c) + 1);
  float2 f0 = __half22float2(h[0]), f1 = __half22float2(h[1]), f2 = __half22float2(h[2]), f3 = __half22float2(h[3]);
  return (f0.x * c0.x + f0.y * c0.y) + (f1.x * c0.z + f1.y * c0.w) + (f2.x * c1.x + f2.y * c1.y) +
         (f3.x * c1.z + f3.y * c1.w);
}

// e = inv c: one block of four warps per row, every thread with its share
// of the row's 16-byte loads (8 FP16 entries each) in flight at once, FP32
// products with c (read through L1), block sum.  The inverse is read with
// an evict-last L2 policy (the SpMV's matrix stream is evict-first), so it
// stays in L2 from one flexible-CG iteration to the next.
constexpr int kMvThreads = 128;
template <class VT>
__global__ void __launch_bounds__(kMvThreads) k_coarse_mv(int nc, int ld, const __half* __restrict__ inv, float rscale,
                                                          const float* __restrict__ c, VT* __restrict__ e,
                                                          const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  const int row = blockIdx.x;
  const int nv8 = nc >> 3, tail = nc & 7;  // whole 8-entry groups inside the row, then a tail
  const uint4* ir = reinterpret_cast<const uint4*>(inv + (size_t)row * ld);
  const unsigned long long keep = l2_evict_last();
  float s[4] = {0.f, 0.f, 0.f, 0.f};
  int k = threadIdx.x;
  for (; k + 3 * kMvThreads < nv8; k += 4 * kMvThreads) {
    uint4 q[4];
#pragma unroll
    for (int u = 0; u < 4; u++) q[u] = ldg_hint(ir + k + u * kMvThreads, keep);
#pragma unroll
    for (int u = 0; u < 4; u++) s[u] += dot8(q[u], c + 8 * (k + u * kMvThreads));
  }
  for (; k < nv8; k += kMvThreads) s[0] += dot8(ldg_hint(ir + k, keep), c + 8 * k);
  if (threadIdx.x < tail) s[1] += __half2float(inv[(size_t)row * ld + 8 * nv8 + threadIdx.x]) * c[8 * nv8 + threadIdx.x];
  float t = warp_sum((s[0] + s[1]) + (s[2] + s[3]));
  __shared__ float sw[kMvThreads / 32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    float tot = 0.f;
#pragma unroll
    for (int w = 0; w < kMvThreads / 32; w++) tot += sw[w];
    e[row] = (VT)(tot * rscale);
  }
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
  // shared memory: G groups x fd[0] partials (G = 1 once fd[0] exceeds the block)
  if (a.fd[0] > 4096) return cudaErrorInvalidValue;
  for (int ax = 1; ax < 3; ax++) {  // support lines of a coarse pair: at most (2 h + 1)^2
    const double h = a.cd[ax] > 1 ? (double)(a.fd[ax] - 1) / (a.cd[ax] - 1) : 1.0;
    if (h > 15.0) return cudaErrorInvalidValue;
  }
  const int G = a.fd[0] <= kRestrictThreads ? kRestrictThreads / a.fd[0] : 1;
  const size_t sm = (size_t)G * a.fd[0] * sizeof(double);
  return launch_k(a.pdl != 0, k_restrict<VT>, dim3(a.cd[1] * a.cd[2]), dim3(kRestrictThreads), sm, s, a, r, c, done);
}

template <class VT>
cudaError_t launch_coarse_solve(const CoarseArgs<VT>& a, const float* c, VT* e, const int* done, cudaStream_t s) {
  if (a.ldinv % 8 || a.ldinv < a.nc) return cudaErrorInvalidValue;
  return launch_k(a.pdl != 0, k_coarse_mv<VT>, dim3(a.nc), dim3(kMvThreads), 0, s, a.nc, a.ldinv, a.inv16,
                  (float)(1.0 / a.inv_scale), c, e, done);
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
