// One-time operator assembly on the device (step0 and calculateZ_CUSP of the
// reference, blascoCodinaHuerta.cpp:3127-3315 and CUDAcodes.cu:281-411).
//
// k_assemble: one element per block iteration.  The Jacobian of the
//   trilinear corner map, its adjugate inverse and detJ are recomputed per
//   Gauss point from the 8 corner coordinates (blascoCodinaHuerta.cpp:
//   2566-2615), so no per-Gauss-point geometry is stored in HBM.  Element
//   blocks Ke (27x27), Ge_d (27x8) and the row sums of Me are added into
//   their CSR slots with FP64 atomics; the slot is found by binary search in
//   the sorted CSR row, so no element colouring and no slot map is needed.
//   In deterministic mode the host launches one colour at a time (no two
//   elements of a colour share a node) and the blocks add without atomics,
//   in the same order every run.
// k_build_z: Z = sum_d G_d^T diag(MdOrigInv) G_d in gather form, one warp
//   per Z row: for every velocity node v of G^T row p (ascending), the lanes
//   take the columns q of G row v and add (G_d[v][q]*Minv[v]) * G_d[v][p] to
//   a shared accumulator of row p.  Lanes of one v never collide, so the
//   accumulation order is fixed (deterministic, ascending v as in the oracle).
#include <cstdio>

#include "kernels.h"

namespace cfd {

namespace {

// Jacobian data of Gauss point k from corner coordinates X[8][3]:
// J[i][j] = sum_m dSp[i][k][m] X[m][j]; returns detJ, writes adj(J)/detJ.
template <class T>
__device__ __forceinline__ T jacobian_inv(const T (*X)[3], const Basis* __restrict__ B, int k, T iJ[3][3]) {
  T J[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T s = 0;
#pragma unroll
      for (int m = 0; m < 8; m++) s += (T)B->dSp[i][k][m] * X[m][j];
      J[i][j] = s;
    }
  T det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) + J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  T inv = T(1) / det;
  iJ[0][0] = (J[1][1] * J[2][2] - J[2][1] * J[1][2]) * inv;
  iJ[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) * inv;
  iJ[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * inv;
  iJ[1][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]) * inv;
  iJ[1][1] = (J[2][2] * J[0][0] - J[2][0] * J[0][2]) * inv;
  iJ[1][2] = -(J[1][2] * J[0][0] - J[1][0] * J[0][2]) * inv;
  iJ[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * inv;
  iJ[2][1] = -(J[2][1] * J[0][0] - J[2][0] * J[0][1]) * inv;
  iJ[2][2] = (J[1][1] * J[0][0] - J[1][0] * J[0][1]) * inv;
  return det;
}

constexpr int kAsmThreads = 128;

__global__ void __launch_bounds__(kAsmThreads) k_assemble(AsmArgs a) {
  __shared__ double sSv[kMaxNGP][27];
  __shared__ double sSp[kMaxNGP][8];
  __shared__ double X[8][3];
  __shared__ int lt[27];
  __shared__ double iJ[kMaxNGP][3][3];
  __shared__ double wd[kMaxNGP];
  __shared__ double gd[kMaxNGP][27][3];
  const int t = threadIdx.x, ngp = a.ngp;
  const Basis* B = a.basis;
  for (int i = t; i < ngp * 27; i += blockDim.x) sSv[i / 27][i % 27] = B->Sv[i / 27][i % 27];
  for (int i = t; i < ngp * 8; i += blockDim.x) sSp[i / 8][i % 8] = B->Sp[i / 8][i % 8];
  for (int pos = a.e_begin + blockIdx.x; pos < a.e_end; pos += gridDim.x) {
    const int e = a.elist ? a.elist[pos] : pos;
    __syncthreads();
    if (t < 27) lt[t] = a.ltog[(size_t)e * 27 + t];
    __syncthreads();
    if (t < 24) X[t / 3][t % 3] = a.coord[3 * (size_t)lt[t / 3] + t % 3];
    __syncthreads();
    if (t < ngp) {
      double J[3][3];
      double det = jacobian_inv<double>(X, B, t, J);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) iJ[t][i][j] = J[i][j];
      wd[t] = det * B->w[t];
    }
    __syncthreads();
    for (int idx = t; idx < ngp * 27; idx += blockDim.x) {
      int k = idx / 27, j = idx % 27;
      double r0 = B->dSv[0][k][j], r1 = B->dSv[1][k][j], r2 = B->dSv[2][k][j];
      for (int i = 0; i < 3; i++) gd[k][j][i] = iJ[k][i][0] * r0 + iJ[k][i][1] * r1 + iJ[k][i][2] * r2;
    }
    __syncthreads();
    // Ke and row sums of Me
    for (int idx = t; idx < 729 + 27; idx += blockDim.x) {
      if (idx < 729) {
        int i = idx / 27, j = idx % 27;
        double s = 0;
        for (int k = 0; k < ngp; k++)
          s += a.viscosity * (gd[k][i][0] * gd[k][j][0] + gd[k][i][1] * gd[k][j][1] + gd[k][i][2] * gd[k][j][2]) *
               wd[k];
        int row = lt[i], col = lt[j];
        int slot = bsearch_slot(a.k_col, a.k_rp[row], a.k_rp[row + 1], col);
        if (slot >= 0) {
          if (a.plain)
            a.kval[slot] += s;
          else
            atomicAdd(a.kval + slot, s);
        }
      } else {
        int i = idx - 729;
        double s = 0;
        for (int j = 0; j < 27; j++) {
          double mij = 0;
          for (int k = 0; k < ngp; k++) mij += sSv[k][i] * sSv[k][j] * wd[k];
          s += mij;
        }
        if (a.plain)
          a.msum[lt[i]] += s;
        else
          atomicAdd(a.msum + lt[i], s);
      }
    }
    // Ge_d[i][m] = -(1/rho) sum_k Sp[k][m] dSv_i/dx_d detJ w
    for (int idx = t; idx < 216; idx += blockDim.x) {
      int i = idx / 8, m = idx % 8;
      double s0 = 0, s1 = 0, s2 = 0;
      for (int k = 0; k < ngp; k++) {
        double f = a.inv_density * sSp[k][m];
        s0 -= f * gd[k][i][0] * wd[k];
        s1 -= f * gd[k][i][1] * wd[k];
        s2 -= f * gd[k][i][2] * wd[k];
      }
      int row = lt[i], col = lt[m];
      int slot = bsearch_slot(a.g_col, a.g_rp[row], a.g_rp[row + 1], col);
      if (slot >= 0) {
        if (a.plain) {
          a.g1[slot] += s0;
          a.g2[slot] += s1;
          a.g3[slot] += s2;
        } else {
          atomicAdd(a.g1 + slot, s0);
          atomicAdd(a.g2 + slot, s1);
          atomicAdd(a.g3 + slot, s2);
        }
      }
    }
  }
}

__global__ void k_fill_gt(long long nnz, const int* __restrict__ pos, const double* __restrict__ g1,
                          const double* __restrict__ g2, const double* __restrict__ g3, double* gt1, double* gt2,
                          double* gt3) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnz; i += (long long)gridDim.x * blockDim.x) {
    int p = pos[i];
    gt1[i] = g1[p];
    gt2[i] = g2[p];
    gt3[i] = g3[p];
  }
}

__global__ void k_md_finalize(int NN, const double* __restrict__ msum, const unsigned char* __restrict__ bc,
                              double* minv_orig, double* minv_free) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += gridDim.x * blockDim.x) {
    double inv = 1.0 / msum[i];
    minv_orig[i] = inv;
    minv_free[i] = bc[i] ? 0.0 : inv;
  }
}

__device__ __forceinline__ int bsearch_smem(const int* col, int n, int key) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int c = col[mid];
    if (c == key) return mid;
    if (c < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

constexpr int kZWarps = 4;

__global__ void __launch_bounds__(32 * kZWarps) k_build_z(ZArgs a) {
  extern __shared__ unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int stride = a.maxrow;
  double* acc = reinterpret_cast<double*>(smem) + (size_t)w * 3 * stride;
  int* cols = reinterpret_cast<int*>(reinterpret_cast<double*>(smem) + (size_t)kZWarps * 3 * stride) + (size_t)w * stride;
  for (int p = blockIdx.x * kZWarps + w; p < a.NNp; p += gridDim.x * kZWarps) {
    const int zb = a.z_rp[p], len = a.z_rp[p + 1] - zb;
    for (int i = lane; i < len; i += 32) {
      cols[i] = a.z_col[zb + i];
      acc[i] = 0.0;
      acc[stride + i] = 0.0;
      acc[2 * stride + i] = 0.0;
    }
    __syncwarp();
    for (int t = a.gt_rp[p]; t < a.gt_rp[p + 1]; t++) {
      const int v = a.gt_col[t];
      const double m = a.minv_orig[v];
      const double p1 = a.gt1[t], p2 = a.gt2[t], p3 = a.gt3[t];
      for (int j = a.g_rp[v] + lane; j < a.g_rp[v + 1]; j += 32) {
        int pos = bsearch_smem(cols, len, a.g_col[j]);
        if (pos >= 0) {
          acc[pos] += (a.g1[j] * m) * p1;
          acc[stride + pos] += (a.g2[j] * m) * p2;
          acc[2 * stride + pos] += (a.g3[j] * m) * p3;
        }
      }
      __syncwarp();
    }
    for (int i = lane; i < len; i += 32) {
      double z = (acc[i] + acc[stride + i]) + acc[2 * stride + i];
      if (cols[i] == p) {
        if (p == a.zeroP && a.zeroP > 0) z *= 1000.0;  // blascoCodinaHuerta.cpp:4167-4180
        a.zdiag[p] = z;
      }
      a.zval[zb + i] = z;
    }
    __syncwarp();
  }
}

__global__ void k_to_float(long long n, const double* __restrict__ in, float* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void k_recip(long long n, const double* __restrict__ in, double* out64, float* out32) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double r = 1.0 / in[i];
    if (out64) out64[i] = r;
    if (out32) out32[i] = (float)r;
  }
}

inline int grid_for(long long n, int threads, int cap = 148 * 32) {
  long long g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

}  // namespace

cudaError_t launch_assemble(const AsmArgs& a, int num_sms, cudaStream_t s) {
  const int ne = a.e_end - a.e_begin;
  if (ne <= 0) return cudaSuccess;
  int grid = ne < num_sms * 16 ? ne : num_sms * 16;
  k_assemble<<<grid, kAsmThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_fill_gt(long long nnz, const int* pos, const double* g1, const double* g2, const double* g3,
                           double* gt1, double* gt2, double* gt3, cudaStream_t s) {
  k_fill_gt<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, pos, g1, g2, g3, gt1, gt2, gt3);
  return cudaGetLastError();
}

cudaError_t launch_md_finalize(int NN, const double* msum, const unsigned char* bcmask, double* minv_orig,
                               double* minv_free, cudaStream_t s) {
  k_md_finalize<<<grid_for(NN, 256), 256, 0, s>>>(NN, msum, bcmask, minv_orig, minv_free);
  return cudaGetLastError();
}

cudaError_t launch_build_z(const ZArgs& a, cudaStream_t s) {
  size_t smem = (size_t)kZWarps * a.maxrow * (3 * sizeof(double) + sizeof(int));
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_build_z, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  int grid = grid_for(a.NNp, kZWarps, 148 * 64);
  k_build_z<<<grid, 32 * kZWarps, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_to_float(long long n, const double* in, float* out, cudaStream_t s) {
  k_to_float<<<grid_for(n, 256), 256, 0, s>>>(n, in, out);
  return cudaGetLastError();
}

cudaError_t launch_recip(long long n, const double* in, double* out64, float* out32, cudaStream_t s) {
  k_recip<<<grid_for(n, 256), 256, 0, s>>>(n, in, out64, out32);
  return cudaGetLastError();
}

}  // namespace cfd
