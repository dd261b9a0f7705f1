// Jacobi-preconditioned CG on the pressure Schur operator Z as one
// persistent cooperative kernel per solve (replaces cusp::krylov::cg with
// precond::diagonal, CUDAcodes.cu:418-451, and MKL dcg, blascoCodinaHuerta.cpp:
// 3981-4055).
//
// Z is stored SELL-32; thread g owns rows g, g+T, g+2T, ... (T = all
// threads, a multiple of 32, so a warp always owns whole slices).  The
// search-direction update p = z + beta p is folded into the next SpMV, which
// evaluates q = Z (z + beta p_old) from gathers of z and p_old and writes
// p_new for its own rows into the other half of a double buffer.  That leaves
// two grid-wide reductions per iteration:
//   A: p_new = z + beta p_old, q = Z p_new (own rows), partial p_new.q  -> reduce
//   B: x += alpha p_new, r -= alpha q, z = Dinv r, partial r.r, r.z     -> reduce
// Each reduction writes per-block partials, passes a bounded grid barrier,
// and every block sums all partials in the same fixed order (FP64), so every
// block takes the same decisions.  Vectors written inside the kernel are
// gathered with L2 loads (ld.cg); the matrix is streamed (ld.cs) so the
// vectors stay resident in L2.  Stopping rule: ||r||_2 <= rtol ||b||_2 on the
// recursively updated residual, checked after each update (as the oracle).
#include <algorithm>

#include "kernels.h"

namespace cfd {

namespace {

constexpr int kPcgThreads = 256;

template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double* part, int phase, unsigned* bar, int* err,
                                            unsigned long long timeout_ns) {
  __shared__ double res[NV];
  const int G = gridDim.x;
  double* buf = part + (size_t)(phase & 1) * 3 * G;
  block_sum<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) buf[(size_t)k * G + blockIdx.x] = v[k];
  if (!grid_barrier(bar, err, timeout_ns)) return false;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double s = 0;
      for (int i = lane; i < G; i += 32) s += __ldcg(buf + (size_t)k * G + i);
      s = warp_sum(s);
      if (lane == 0) res[k] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = res[k];
  __syncthreads();
  return true;
}

template <class VT>
__global__ void __launch_bounds__(kPcgThreads, 5) k_pcg(PcgArgs<VT> a) {
  const int T = gridDim.x * blockDim.x;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.n;
  VT* P0 = a.p;
  VT* P1 = a.p + n;
  int phase = 0;

  // ---- initial residual ----
  double v3[3] = {0, 0, 0};
  for (int i = g; i < n; i += T) {
    const double bi = (double)a.b[i];
    double ri = bi;
    if (a.warm) {
      const int s = i >> 5, l = i & 31;
      const int b = __ldg(a.off + s) + l, w = (__ldg(a.off + s + 1) - __ldg(a.off + s)) >> 5;
      VT q = 0;
      for (int j = 0; j < w; j++) q += __ldcs(a.val + b + 32 * j) * a.x[__ldcs(a.col + b + 32 * j)];
      ri = bi - (double)q;
    } else {
      a.x[i] = (VT)0;
    }
    const VT rv = (VT)ri;
    const VT zv = (VT)((double)rv * (double)a.dinv[i]);
    a.r[i] = rv;
    a.z[i] = zv;
    P0[i] = (VT)0;
    v3[0] += bi * bi;
    v3[1] += (double)rv * (double)zv;
    v3[2] += (double)rv * (double)rv;
  }
  const bool alive = grid_reduce<3>(v3, a.part, phase++, a.bar, a.err, a.timeout_ns);
  const double bnorm = sqrt(v3[0]);
  double rz = v3[1];
  double rn = sqrt(v3[2]);
  const double tol = a.rtol * bnorm;
  int its = 0, status = 1;
  if (!alive) {
    status = 3;
  } else if (!isfinite(bnorm) || !isfinite(rn)) {
    status = 2;
  } else if (bnorm == 0.0) {
    for (int i = g; i < n; i += T) a.x[i] = (VT)0;
    status = 0;
    rn = 0;
  } else if (rn <= tol) {
    status = 0;
  } else {
    VT beta = 0;
    VT* pold = P0;
    VT* pnew = P1;
    while (its < a.maxit) {
      // A: p_new = z + beta p_old;  q = Z p_new
      double pq = 0;
      for (int i = g; i < n; i += T) {
        const int s = i >> 5, l = i & 31;
        const int b = __ldg(a.off + s) + l, w = (__ldg(a.off + s + 1) - __ldg(a.off + s)) >> 5;
        VT q = 0;
#pragma unroll 4
        for (int j = 0; j < w; j++) {
          const int c = __ldcs(a.col + b + 32 * j);
          const VT pc = __ldcg(a.z + c) + beta * __ldcg(pold + c);
          q += __ldcs(a.val + b + 32 * j) * pc;
        }
        const VT pi = a.z[i] + beta * pold[i];
        pnew[i] = pi;
        a.q[i] = q;
        pq += (double)pi * (double)q;
      }
      double v1[1] = {pq};
      if (!grid_reduce<1>(v1, a.part, phase++, a.bar, a.err, a.timeout_ns)) { status = 3; break; }
      const double alpha = rz / v1[0];
      // B: updates on own rows
      double v2[2] = {0, 0};
      for (int i = g; i < n; i += T) {
        const double pi = (double)pnew[i], qi = (double)a.q[i];
        a.x[i] = (VT)((double)a.x[i] + alpha * pi);
        const VT rv = (VT)((double)a.r[i] - alpha * qi);
        const VT zv = (VT)((double)rv * (double)a.dinv[i]);
        a.r[i] = rv;
        a.z[i] = zv;
        v2[0] += (double)rv * (double)rv;
        v2[1] += (double)rv * (double)zv;
      }
      if (!grid_reduce<2>(v2, a.part, phase++, a.bar, a.err, a.timeout_ns)) { status = 3; break; }
      its++;
      rn = sqrt(v2[0]);
      if (!isfinite(rn)) { status = 2; break; }
      if (rn <= tol) { status = 0; break; }
      beta = (VT)(v2[1] / rz);
      rz = v2[1];
      VT* t = pold;
      pold = pnew;
      pnew = t;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.result[0] = its;
    a.result[1] = bnorm > 0 ? rn / bnorm : 0.0;
    a.result[2] = status;
    a.result[3] = bnorm;
  }
}

constexpr int kResThreads = 256;

// r = b - Z x in FP64 (SELL-32 Z), rf = (float) r, per-block partial of r^2.
__global__ void __launch_bounds__(kResThreads) k_residual64(int n, const int* __restrict__ off,
                                                             const int* __restrict__ col,
                                                             const double* __restrict__ val,
                                                             const double* __restrict__ b,
                                                             const double* __restrict__ x, double* r, float* rf,
                                                             double* part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0};
  if (i < n) {
    const int s = i >> 5, l = i & 31;
    const int bb = __ldg(off + s) + l, w = (__ldg(off + s + 1) - __ldg(off + s)) >> 5;
    double q = 0;
#pragma unroll 4
    for (int j = 0; j < w; j++) q += __ldcs(val + bb + 32 * j) * __ldg(x + __ldcs(col + bb + 32 * j));
    const double ri = b[i] - q;
    r[i] = ri;
    if (rf) rf[i] = (float)ri;
    acc[0] = ri * ri;
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

__global__ void k_axpy_f2d(int n, const float* __restrict__ e, double* x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += (double)e[i];
}

__global__ void k_sum_partials(const double* __restrict__ part, int n, double* out) {
  double v[1] = {0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) v[0] += part[i];
  block_sum<1>(v);
  if (threadIdx.x == 0) out[0] = v[0];
}

// Self-test of the bounded wait: one warp watches a flag that nothing sets
// and gives up after timeout_ns, reporting through *err.
__global__ void k_wait_selftest(const int* flag, int* err, unsigned long long timeout_ns) {
  if (threadIdx.x != 0) return;
  unsigned long long t0 = global_ns();
  while (ld_volatile_i32(flag) == 0) {
    if (global_ns() - t0 > timeout_ns) {
      atomicExch(err, 1);
      return;
    }
    __nanosleep(1000);
  }
}

}  // namespace

cudaError_t launch_wait_selftest(const int* flag, int* err, unsigned long long timeout_ns, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(flag, err, timeout_ns);
  return cudaGetLastError();
}

template <class VT>
int pcg_max_grid(int n, int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<VT>, kPcgThreads, 0);
  long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
  long long want = ((long long)n + kPcgThreads - 1) / kPcgThreads;  // one row per thread at most
  if (want < 1) want = 1;
  return (int)std::min(cap, want);
}

template <class VT>
cudaError_t launch_pcg(const PcgArgs<VT>& a, int grid, cudaStream_t s) {
  PcgArgs<VT> args = a;
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel((const void*)k_pcg<VT>, dim3(grid), dim3(kPcgThreads), params, 0, s);
}

int residual_blocks(int n, int) { return std::max(1, (n + kResThreads - 1) / kResThreads); }

cudaError_t launch_residual64(int n, const int* off, const int* col, const double* val, const double* b,
                              const double* x, double* r, float* rf, double* part, int nblocks, cudaStream_t s) {
  k_residual64<<<nblocks, kResThreads, 0, s>>>(n, off, col, val, b, x, r, rf, part);
  return cudaGetLastError();
}

cudaError_t launch_axpy_f2d(int n, const float* e, double* x, cudaStream_t s) {
  int g = std::max(1, std::min((n + 255) / 256, 148 * 8));
  k_axpy_f2d<<<g, 256, 0, s>>>(n, e, x);
  return cudaGetLastError();
}

cudaError_t launch_sum_partials(const double* part, int n, double* out, cudaStream_t s) {
  k_sum_partials<<<1, 1024, 0, s>>>(part, n, out);
  return cudaGetLastError();
}

template int pcg_max_grid<double>(int, int);
template int pcg_max_grid<float>(int, int);
template cudaError_t launch_pcg<double>(const PcgArgs<double>&, int, cudaStream_t);
template cudaError_t launch_pcg<float>(const PcgArgs<float>&, int, cudaStream_t);

}  // namespace cfd
