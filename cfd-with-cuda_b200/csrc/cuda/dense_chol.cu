// Dense SPD inverse on the device, FP64: the coarse matrix Zc = P^T Z P of
// the two-level preconditioner (a few thousand rows) is factored and
// inverted here instead of on the host, and its scaled FP16 copy (the
// operand of the coarse solve in every iteration) is written in place.
//
//   A = L L^T              blocked right-looking Cholesky, 64-wide panels:
//                          diagonal block in one CTA, the panel below it by
//                          a row-wise triangular solve, the trailing lower
//                          triangle updated by 64 x 64 tiles
//   Y = L^-1               blocked forward substitution with the identity
//                          as right-hand side (Y is lower triangular)
//   A^-1 = Y^T Y           64 x 64 tiles of the lower triangle, mirrored
//
// Row-major storage with leading dimension ld (>= n, a multiple of 64), so
// every tile is whole; the padding rows and columns hold the identity and
// stay out of the real rows.  About n^3 / 3 multiply-adds per stage; the
// tile kernels keep a 64 x 64 output tile in registers (4 x 4 per thread)
// and read 64-wide strips of the operands from shared memory.
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace cfd {

namespace {

constexpr int kNB = 64;            // panel and tile width
constexpr int kTileThreads = 256;  // 16 x 16 threads, 4 x 4 outputs each
constexpr int kOneTile = kNB * (kNB + 1) * (int)sizeof(double);  // one padded 64 x 64 tile
using Tile = double[kNB + 1];

// Unblocked Cholesky of the diagonal block at (k0, k0) in shared memory;
// *info = k0 + j + 1 for the first non-positive pivot.
__global__ void __launch_bounds__(kNB * 4) k_chol_diag(double* A, int ld, int k0, int* info) {
  extern __shared__ double dsm[];
  Tile* s = reinterpret_cast<Tile*>(dsm);
  __shared__ double piv;
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    const int i = idx / kNB, j = idx % kNB;
    s[i][j] = A[(size_t)(k0 + i) * ld + k0 + j];
  }
  __syncthreads();
  for (int j = 0; j < kNB; j++) {
    if (threadIdx.x == 0) {
      const double d = s[j][j];
      if (!(d > 0.0) || !isfinite(d)) {
        if (*info == 0) *info = k0 + j + 1;
        piv = 1.0;
      } else {
        piv = sqrt(d);
      }
      s[j][j] = piv;
    }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < kNB; i += blockDim.x) s[i][j] /= piv;
    __syncthreads();
    // trailing update of the block's lower triangle
    const int m = kNB - j - 1;
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
      const int i = j + 1 + idx / m, l = j + 1 + idx % m;
      if (l <= i) s[i][l] -= s[i][j] * s[l][j];
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    const int i = idx / kNB, j = idx % kNB;
    A[(size_t)(k0 + i) * ld + k0 + j] = j <= i ? s[i][j] : 0.0;
  }
}

// Rows below the diagonal block, 64 per CTA: x L_kk^T = a, one thread per
// row, the diagonal block and the rows' strips in shared memory.
__global__ void __launch_bounds__(kNB) k_chol_panel(double* A, int ld, int k0) {
  extern __shared__ double dsm[];
  Tile* L = reinterpret_cast<Tile*>(dsm);
  Tile* X = L + kNB;
  const int r0 = k0 + kNB + blockIdx.x * kNB;
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    const int i = idx / kNB, j = idx % kNB;
    L[i][j] = A[(size_t)(k0 + i) * ld + k0 + j];
    X[i][j] = A[(size_t)(r0 + i) * ld + k0 + j];
  }
  __syncthreads();
  const int t = threadIdx.x;
  for (int j = 0; j < kNB; j++) {
    double v = X[t][j];
    for (int m = 0; m < j; m++) v -= X[t][m] * L[j][m];
    X[t][j] = v / L[j][j];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    const int i = idx / kNB, j = idx % kNB;
    A[(size_t)(r0 + i) * ld + k0 + j] = X[i][j];
  }
}

// Tile (I, J), I >= J, of a lower-triangular tile grid numbered row by row
// (b = I (I + 1) / 2 + J).
__device__ __forceinline__ void lower_tile(int b, int& I, int& J) {
  int i = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= b) i++;
  while (i * (i + 1) / 2 > b) i--;
  I = i;
  J = b - i * (i + 1) / 2;
}

// acc[u][v] += sum_k a_rows[ty + 16u][k] * b_rows[tx + 16v][k] over one
// 64-wide strip (rows of both operands in shared memory)
__device__ __forceinline__ void tile_nt(const Tile* a, const Tile* b, double (&acc)[4][4]) {
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  for (int k = 0; k < kNB; k++) {
    double x[4], y[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      x[u] = a[ty + 16 * u][k];
      y[u] = b[tx + 16 * u][k];
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int v = 0; v < 4; v++) acc[u][v] += x[u] * y[v];
  }
}

// C[I][J] -= P_I P_J^T for the lower tiles of the trailing matrix (rows and
// columns from k1 on), P = the factored panel columns k0 .. k0 + 63.
__global__ void __launch_bounds__(kTileThreads) k_chol_trail(double* A, int ld, int k0, int k1) {
  extern __shared__ double dsm[];
  Tile* PI = reinterpret_cast<Tile*>(dsm);
  Tile* PJ = PI + kNB;
  int I, J;
  lower_tile(blockIdx.x, I, J);
  const int ri = k1 + I * kNB, rj = k1 + J * kNB;
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    const int a = idx / kNB, k = idx % kNB;
    PI[a][k] = A[(size_t)(ri + a) * ld + k0 + k];
    PJ[a][k] = A[(size_t)(rj + a) * ld + k0 + k];
  }
  __syncthreads();
  double acc[4][4] = {};
  tile_nt(PI, PJ, acc);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int r = ri + ty + 16 * u, c = rj + tx + 16 * v;
      if (c <= r) A[(size_t)r * ld + c] -= acc[u][v];
    }
}

// Forward substitution, block row at k0: Y_i = L_ii^-1 B_i for the columns
// below k0 + 64 (B_i is zero beyond), one thread per column.
__global__ void __launch_bounds__(kNB) k_fwd_diag(const double* L, double* Y, int ld, int k0) {
  extern __shared__ double dsm[];
  Tile* Ld = reinterpret_cast<Tile*>(dsm);
  Tile* C = Ld + kNB;  // C[row][thread]
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    const int i = idx / kNB, j = idx % kNB;
    Ld[i][j] = L[(size_t)(k0 + i) * ld + k0 + j];
  }
  const int c = blockIdx.x * kNB + threadIdx.x;
  for (int r = 0; r < kNB; r++) C[r][threadIdx.x] = Y[(size_t)(k0 + r) * ld + c];
  __syncthreads();
  for (int r = 0; r < kNB; r++) {
    double v = C[r][threadIdx.x];
    for (int m = 0; m < r; m++) v -= Ld[r][m] * C[m][threadIdx.x];
    C[r][threadIdx.x] = v / Ld[r][r];
  }
  for (int r = 0; r < kNB; r++) Y[(size_t)(k0 + r) * ld + c] = C[r][threadIdx.x];
}

// Y[rows >= k1][cols < k1] -= L[rows][k0 .. k0+63] Y[k0 .. k0+63][cols]:
// row tile I over the rows below, column tile J over the columns the block
// row reaches (ncol_tiles of them).
__global__ void __launch_bounds__(kTileThreads) k_fwd_update(const double* L, double* Y, int ld, int k0, int k1,
                                                              int ncol_tiles) {
  extern __shared__ double dsm[];
  Tile* Ls = reinterpret_cast<Tile*>(dsm);
  Tile* Yt = Ls + kNB;  // Yt[col][k]: the block row transposed
  const int I = blockIdx.x / ncol_tiles, J = blockIdx.x % ncol_tiles;
  const int ri = k1 + I * kNB, cj = J * kNB;
  for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
    const int a = idx / kNB, k = idx % kNB;
    Ls[a][k] = L[(size_t)(ri + a) * ld + k0 + k];
    Yt[k][a] = Y[(size_t)(k0 + a) * ld + cj + k];
  }
  __syncthreads();
  double acc[4][4] = {};
  tile_nt(Ls, Yt, acc);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) Y[(size_t)(ri + ty + 16 * u) * ld + cj + tx + 16 * v] -= acc[u][v];
}

// inv tile (I, J), I >= J: sum over rows i >= 64 I of Y[i][a] Y[i][b]
// (Y lower triangular), written to both triangles.
__global__ void __launch_bounds__(kTileThreads) k_yty(const double* Y, double* inv, int ld, int ntiles) {
  extern __shared__ double dsm[];
  Tile* YA = reinterpret_cast<Tile*>(dsm);  // YA[col][row]: columns of the strip
  Tile* YB = YA + kNB;
  int I, J;
  lower_tile(blockIdx.x, I, J);
  const int ca = I * kNB, cb = J * kNB;
  double acc[4][4] = {};
  for (int t = I; t < ntiles; t++) {
    const int r0 = t * kNB;
    __syncthreads();
    for (int idx = threadIdx.x; idx < kNB * kNB; idx += blockDim.x) {
      const int i = idx / kNB, c = idx % kNB;
      YA[c][i] = Y[(size_t)(r0 + i) * ld + ca + c];
      YB[c][i] = Y[(size_t)(r0 + i) * ld + cb + c];
    }
    __syncthreads();
    tile_nt(YA, YB, acc);
  }
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int r = ca + ty + 16 * u, c = cb + tx + 16 * v;
      inv[(size_t)r * ld + c] = acc[u][v];
      inv[(size_t)c * ld + r] = acc[u][v];
    }
}

// rows and columns n .. ld-1 become the identity, so the padded matrix stays
// SPD and its factor and inverse stay block diagonal
__global__ void k_identity_pad(double* A, int n, int ld) {
  const long long total = (long long)ld * ld;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / ld), j = (int)(idx % ld);
    if (i >= n || j >= n) A[idx] = i == j ? 1.0 : 0.0;
  }
}

__global__ void k_identity(double* Y, int ld) {
  const long long total = (long long)ld * ld;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x)
    Y[idx] = idx / ld == idx % ld ? 1.0 : 0.0;
}

__global__ void k_absmax(const double* A, int n, int ld, unsigned long long* out) {
  double m = 0.0;
  const long long total = (long long)n * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(A[(idx / n) * ld + idx % n]));
  m = warp_max(m);
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_to_half(const double* A, int n, int ld, const unsigned long long* amax, int ldh, __half* out) {
  const double am = __longlong_as_double((long long)*amax);
  const double scale = am > 0 ? 16384.0 / am : 1.0;
  const long long total = (long long)n * ldh;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / ldh), j = (int)(idx % ldh);
    out[idx] = __float2half(j < n ? (float)(A[(size_t)i * ld + j] * scale) : 0.f);
  }
}

int grid_for(long long total) {
  const long long g = (total + 255) / 256;
  return (int)(g > 148 * 32 ? 148 * 32 : (g < 1 ? 1 : g));
}

}  // namespace

int spd_inverse_ld(int n) { return (n + kNB - 1) / kNB * kNB; }

cudaError_t spd_inverse_device(double* A, double* work, int n, int ld, int* info, cudaStream_t s) {
  if (n < 1 || ld < n || ld % kNB) return cudaErrorInvalidValue;
  const int T = ld / kNB;
  cudaError_t e = cudaSuccess;
  const void* two_tiles[] = {(const void*)k_chol_panel, (const void*)k_chol_trail, (const void*)k_fwd_diag,
                             (const void*)k_fwd_update, (const void*)k_yty};
  for (const void* f : two_tiles)
    if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kOneTile)) != cudaSuccess)
      return e;
  if ((e = cudaMemsetAsync(info, 0, sizeof(int), s)) != cudaSuccess) return e;
  k_identity_pad<<<grid_for((long long)ld * ld), 256, 0, s>>>(A, n, ld);
  // Cholesky
  for (int t = 0; t < T; t++) {
    const int k0 = t * kNB, k1 = k0 + kNB, rest = T - t - 1;
    k_chol_diag<<<1, kNB * 4, kOneTile, s>>>(A, ld, k0, info);
    if (rest > 0) {
      k_chol_panel<<<rest, kNB, 2 * kOneTile, s>>>(A, ld, k0);
      k_chol_trail<<<rest * (rest + 1) / 2, kTileThreads, 2 * kOneTile, s>>>(A, ld, k0, k1);
    }
  }
  // Y = L^-1 in work
  k_identity<<<grid_for((long long)ld * ld), 256, 0, s>>>(work, ld);
  for (int t = 0; t < T; t++) {
    const int k0 = t * kNB, k1 = k0 + kNB, rest = T - t - 1;
    k_fwd_diag<<<t + 1, kNB, 2 * kOneTile, s>>>(A, work, ld, k0);
    if (rest > 0) k_fwd_update<<<rest * (t + 1), kTileThreads, 2 * kOneTile, s>>>(A, work, ld, k0, k1, t + 1);
  }
  // A^-1 = Y^T Y into A
  k_yty<<<T * (T + 1) / 2, kTileThreads, 2 * kOneTile, s>>>(work, A, ld, T);
  return cudaGetLastError();
}

cudaError_t spd_inverse_to_half(const double* inv, int n, int ld, unsigned long long* amax_bits, int ldh, __half* out,
                                cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(amax_bits, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  k_absmax<<<grid_for((long long)n * n), 256, 0, s>>>(inv, n, ld, amax_bits);
  k_to_half<<<grid_for((long long)n * ldh), 256, 0, s>>>(inv, n, ld, amax_bits, ldh, out);
  return cudaGetLastError();
}

}  // namespace cfd
