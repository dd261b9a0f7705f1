// Jacobi-preconditioned CG on the pressure Schur operator Z as one
// persistent cooperative kernel per solve (replaces cusp::krylov::cg with
// precond::diagonal, CUDAcodes.cu:418-451, and MKL dcg, blascoCodinaHuerta.cpp:
// 3981-4055).
//
// Each warp owns a contiguous block of rows.  Per iteration:
//   A: q = Z p on own rows (one warp per row), partial p.q      -> grid reduce
//   B: x += a p, r -= a q, z = Dinv r, partial r.r and r.z      -> grid reduce
//   C: p = z + b p on own rows                                  -> grid barrier
// Grid reductions write per-block partials, pass a bounded grid barrier, and
// every block sums all partials in the same fixed order (FP64), so all blocks
// take identical decisions and results do not depend on timing.  Stopping
// rule: ||r||_2 <= rtol ||b||_2 on the recursively updated residual, checked
// after each update, exactly as the CPU oracle.
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
__global__ void __launch_bounds__(kPcgThreads) k_pcg(PcgArgs<VT> a) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const long long gw = (long long)blockIdx.x * wpb + wib, nw = (long long)gridDim.x * wpb;
  const int n = a.n;
  const int r0 = (int)(n * gw / nw), r1 = (int)(n * (gw + 1) / nw);
  int phase = 0;
  bool alive = true;

  // ---- initial residual ----
  if (a.warm) {
    for (int i = r0; i < r1; i++) {
      double s = 0;
      for (int j = a.rp[i] + lane; j < a.rp[i + 1]; j += 32) s += (double)a.val[j] * (double)a.x[a.col[j]];
      s = warp_sum(s);
      if (lane == 0) a.q[i] = (VT)s;
    }
    __syncwarp();
  }
  double v3[3] = {0, 0, 0};
  for (int i = r0 + lane; i < r1; i += 32) {
    double bi = (double)a.b[i];
    double ri = a.warm ? bi - (double)a.q[i] : bi;
    if (!a.warm) a.x[i] = (VT)0;
    double zi = ri * (double)a.dinv[i];
    a.r[i] = (VT)ri;
    a.z[i] = (VT)zi;
    a.p[i] = (VT)zi;
    v3[0] += bi * bi;
    v3[1] += ri * (double)(VT)zi;
    v3[2] += ri * ri;
  }
  alive = grid_reduce<3>(v3, a.part, phase++, a.bar, a.err, a.timeout_ns);
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
    for (int i = r0 + lane; i < r1; i += 32) a.x[i] = (VT)0;
    status = 0;
    rn = 0;
  } else if (rn <= tol) {
    status = 0;
  } else {
    while (its < a.maxit) {
      // A: q = Z p
      double pq = 0;
      for (int i = r0; i < r1; i++) {
        VT s = 0;
        const int b = __ldg(a.rp + i), e = __ldg(a.rp + i + 1);
        for (int j = b + lane; j < e; j += 32) s += __ldg(a.val + j) * __ldcg(a.p + __ldg(a.col + j));
        s = warp_sum(s);
        if (lane == 0) {
          a.q[i] = s;
          pq += (double)a.p[i] * (double)s;
        }
      }
      double v1[1] = {pq};
      if (!grid_reduce<1>(v1, a.part, phase++, a.bar, a.err, a.timeout_ns)) { status = 3; break; }
      const double alpha = rz / v1[0];
      // B: updates
      double v2[2] = {0, 0};
      for (int i = r0 + lane; i < r1; i += 32) {
        double pi = (double)a.p[i], qi = (double)__ldcg(a.q + i);
        a.x[i] = (VT)((double)a.x[i] + alpha * pi);
        double ri = (double)a.r[i] - alpha * qi;
        VT rv = (VT)ri;
        VT zv = (VT)((double)rv * (double)a.dinv[i]);
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
      const double beta = v2[1] / rz;
      rz = v2[1];
      // C: p = z + beta p
      for (int i = r0 + lane; i < r1; i += 32) a.p[i] = (VT)((double)a.z[i] + beta * (double)a.p[i]);
      if (!grid_barrier(a.bar, a.err, a.timeout_ns)) { status = 3; break; }
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

// r = b - Z x in FP64, rf = (float) r, per-block partial of r^2.
__global__ void __launch_bounds__(kResThreads) k_residual64(int n, const int* __restrict__ rp,
                                                             const int* __restrict__ col,
                                                             const double* __restrict__ val,
                                                             const double* __restrict__ b,
                                                             const double* __restrict__ x, double* r, float* rf,
                                                             double* part) {
  const int lane = threadIdx.x & 31;
  const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0};
  for (long long i = gw; i < n; i += nw) {
    double s = 0;
    for (int j = rp[i] + lane; j < rp[i + 1]; j += 32) s += __ldg(val + j) * __ldg(x + __ldg(col + j));
    s = warp_sum(s);
    if (lane == 0) {
      double ri = b[i] - s;
      r[i] = ri;
      if (rf) rf[i] = (float)ri;
      acc[0] += ri * ri;
    }
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
  // about 8 rows per warp at least, so that small systems use few blocks
  long long want = ((long long)n + (kPcgThreads / 32) * 8 - 1) / ((kPcgThreads / 32) * 8);
  if (want < 1) want = 1;
  return (int)std::min(cap, want);
}

template <class VT>
cudaError_t launch_pcg(const PcgArgs<VT>& a, int grid, cudaStream_t s) {
  PcgArgs<VT> args = a;
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel((const void*)k_pcg<VT>, dim3(grid), dim3(kPcgThreads), params, 0, s);
}

int residual_blocks(int n, int num_sms) {
  long long g = ((long long)n + (kResThreads / 32) - 1) / (kResThreads / 32);
  return (int)std::max(1LL, std::min(g, (long long)num_sms * 8));
}

cudaError_t launch_residual64(int n, const int* rp, const int* col, const double* val, const double* b,
                              const double* x, double* r, float* rf, double* part, int nblocks, cudaStream_t s) {
  k_residual64<<<nblocks, kResThreads, 0, s>>>(n, rp, col, val, b, x, r, rf, part);
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
