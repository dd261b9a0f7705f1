// Galerkin coarse matrix of the two-level pressure preconditioners on the
// device: W = Z P row by row, then Zc = P^T W, dense, symmetrised.  P holds
// the trilinear hat functions of the coarse lattice (hat tables i0, f per
// axis, as the host build makes them in coarse.cpp); Z is the assembled
// pressure matrix in CSR.
//
// Every sum is taken in the host build's order with the same fused
// multiply-adds, so on an identity-numbered grid (pressure node = voxel)
// the matrix is bit-identical to coarse_build's: W row p adds its CSR
// entries in row order, corner by corner; Zc(i, j) adds the fine nodes of
// the support of hat i in ascending order.
#include "common.cuh"
#include "kernels.h"

namespace cfd {

namespace {

// weight of coarse node i along one axis at fine coordinate x
__device__ __forceinline__ double hat_weight(const int* i0, const double* f, int x, int i) {
  const int k = i0[x];
  return k == i ? 1.0 - f[x] : (k + 1 == i ? f[x] : 0.0);
}

// One thread per pressure row p: the coarse box its columns reach (at most
// 3 nodes per axis, else *bad is set and the row left empty) and the 27
// coefficients of W = Z P over that box.
__global__ void __launch_bounds__(128) k_galerkin_w(GalerkinArgs g) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.np) return;
  const int fx = g.fd[0], fxy = g.fd[0] * g.fd[1];
  const int r0 = g.rp[p], r1 = g.rp[p + 1];
  int mn[3] = {1 << 30, 1 << 30, 1 << 30}, mx[3] = {-1, -1, -1};
  for (int k = r0; k < r1; k++) {
    const int q = g.col[k];
    const int v = g.vox ? g.vox[q] : q;
    const int i[3] = {g.i0x[v % fx], g.i0y[(v / fx) % g.fd[1]], g.i0z[v / fxy]};
    for (int a = 0; a < 3; a++) {
      mn[a] = min(mn[a], i[a]);
      mx[a] = max(mx[a], min(i[a] + 1, g.cd[a] - 1));
    }
  }
  bool wide = false;
  for (int a = 0; a < 3; a++) {
    if (mx[a] < mn[a]) mx[a] = mn[a] = 0;
    wide |= mx[a] - mn[a] + 1 > 3;
  }
  double w[27];
#pragma unroll
  for (int t = 0; t < 27; t++) w[t] = 0.0;
  if (wide) {
    atomicExch(g.bad, 1);
  } else {
    for (int k = r0; k < r1; k++) {
      const int q = g.col[k];
      const int v = g.vox ? g.vox[q] : q;
      const int x = v % fx, y = (v / fx) % g.fd[1], z = v / fxy;
      const int ix = g.i0x[x], iy = g.i0y[y], iz = g.i0z[z];
      const double wx = g.fx[x], wy = g.fy[y], wz = g.fz[z];
      const double val = g.val[k];
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        if ((dx && g.cd[0] < 2) || (dy && g.cd[1] < 2) || (dz && g.cd[2] < 2)) continue;
        const double wt = __dmul_rn(__dmul_rn(dx ? wx : 1.0 - wx, dy ? wy : 1.0 - wy), dz ? wz : 1.0 - wz);
        if (wt == 0.0) continue;
        const int t = (ix + dx - mn[0]) + 3 * (iy + dy - mn[1]) + 9 * (iz + dz - mn[2]);
        w[t] = __fma_rn(val, wt, w[t]);
      }
    }
  }
  double* wr = g.w27 + 27 * (size_t)p;
  for (int t = 0; t < 27; t++) wr[t] = w[t];
  g.wlo[p] = wide ? 0 : mn[0] + g.cd[0] * (mn[1] + g.cd[1] * mn[2]);
  if (g.zp && !wide)
    for (int t = 0; t < 27; t++) g.zp[((size_t)(p >> 5) * 27 + t) * 32 + (p & 31)] = (float)w[t];
}

// One block per coarse node i, one thread per coarse offset (dx, dy, dz) in
// [-2, 2]^3: Zc(i, j) = sum over the fine nodes of the support of hat i, in
// ascending voxel order, of w_i(p) W(p, j).  The support's fine nodes are
// staged 32 at a time (weight, box origin, W row) in shared memory.
constexpr int kZcThreads = 128;
constexpr int kZcChunk = 32;
__global__ void __launch_bounds__(kZcThreads) k_galerkin_zc(GalerkinArgs g) {
  __shared__ double sw[kZcChunk][27];
  __shared__ double swt[kZcChunk];
  __shared__ int sp[kZcChunk], slo[kZcChunk][3];
  const int i = blockIdx.x;
  const int cx = g.cd[0], cy = g.cd[1];
  const int ix = i % cx, iy = (i / cx) % cy, iz = i / (cx * cy);
  const int x0 = g.rx[2 * ix], x1 = g.rx[2 * ix + 1];
  const int y0 = g.ry[2 * iy], y1 = g.ry[2 * iy + 1];
  const int z0 = g.rz[2 * iz], z1 = g.rz[2 * iz + 1];
  const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
  const long long S = (long long)nx * ny * nz;
  const int t = threadIdx.x;
  const int jx = ix + t % 5 - 2, jy = iy + (t / 5) % 5 - 2, jz = iz + t / 25 - 2;
  const bool valid = t < 125 && jx >= 0 && jx < cx && jy >= 0 && jy < cy && jz >= 0 && jz < g.cd[2];
  double acc = 0.0;
  for (long long s0 = 0; s0 < S; s0 += kZcChunk) {
    const int cnt = (int)min((long long)kZcChunk, S - s0);
    __syncthreads();
    if (t < cnt) {
      const long long s = s0 + t;
      const int x = x0 + (int)(s % nx), y = y0 + (int)((s / nx) % ny), z = z0 + (int)(s / ((long long)nx * ny));
      const int v = x + g.fd[0] * (y + g.fd[1] * z);
      const int p = g.pofv ? g.pofv[v] : v;
      sp[t] = p;
      swt[t] = __dmul_rn(__dmul_rn(hat_weight(g.i0x, g.fx, x, ix), hat_weight(g.i0y, g.fy, y, iy)),
                         hat_weight(g.i0z, g.fz, z, iz));
      const int lo = g.wlo[p];
      slo[t][0] = lo % cx;
      slo[t][1] = (lo / cx) % cy;
      slo[t][2] = lo / (cx * cy);
    }
    __syncthreads();
    for (int e = t; e < cnt * 27; e += kZcThreads) sw[e / 27][e % 27] = g.w27[27 * (size_t)sp[e / 27] + e % 27];
    __syncthreads();
    if (valid)
      for (int u = 0; u < cnt; u++) {
        const double wt = swt[u];
        const int bx = jx - slo[u][0], by = jy - slo[u][1], bz = jz - slo[u][2];
        if (wt == 0.0 || bx < 0 || bx > 2 || by < 0 || by > 2 || bz < 0 || bz > 2) continue;
        const double v = sw[u][bx + 3 * by + 9 * bz];
        if (v != 0.0) acc = __fma_rn(wt, v, acc);
      }
  }
  if (valid) g.zc[(size_t)i * g.ld + jx + cx * (jy + cy * jz)] = acc;
}

// The rounding of the two accumulation orders made symmetric:
// Zc(i, j) = Zc(j, i) = (Zc(i, j) + Zc(j, i)) / 2, each pair by the block of
// its larger index.
__global__ void __launch_bounds__(kZcThreads) k_galerkin_sym(GalerkinArgs g) {
  const int i = blockIdx.x;
  const int cx = g.cd[0], cy = g.cd[1];
  const int ix = i % cx, iy = (i / cx) % cy, iz = i / (cx * cy);
  const int t = threadIdx.x;
  const int jx = ix + t % 5 - 2, jy = iy + (t / 5) % 5 - 2, jz = iz + t / 25 - 2;
  if (!(t < 125 && jx >= 0 && jx < cx && jy >= 0 && jy < cy && jz >= 0 && jz < g.cd[2])) return;
  const int j = jx + cx * (jy + cy * jz);
  if (j >= i) return;
  double* a = g.zc + (size_t)i * g.ld + j;
  double* b = g.zc + (size_t)j * g.ld + i;
  const double s = 0.5 * (*a + *b);
  *a = s;
  *b = s;
}

}  // namespace

cudaError_t launch_galerkin(const GalerkinArgs& g, cudaStream_t s) {
  if (g.np < 1 || g.nc < 1) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(g.zc, 0, (size_t)g.nc * g.ld * sizeof(double), s);
  if (e != cudaSuccess) return e;
  if (g.zp) {
    e = cudaMemsetAsync(g.zp, 0, (size_t)((g.np + 31) / 32) * 27 * 32 * sizeof(float), s);
    if (e != cudaSuccess) return e;
  }
  k_galerkin_w<<<(g.np + 127) / 128, 128, 0, s>>>(g);
  k_galerkin_zc<<<g.nc, kZcThreads, 0, s>>>(g);
  k_galerkin_sym<<<g.nc, kZcThreads, 0, s>>>(g);
  return cudaGetLastError();
}

}  // namespace cfd
