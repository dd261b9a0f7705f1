// Jacobi-preconditioned CG on a caller-provided CSR system that allocates
// no device memory: cfd_pcg_solve_noalloc.
//
// Who needs it: callers that cannot call cudaMalloc/cudaFree while they run
// the pressure solve.  A coupled multi-physics code that keeps other streams
// busy cannot afford cudaFree, which synchronizes the whole device; a host
// application that reserves all of its device memory up front through its
// own pool allocator cannot let a library allocate at solve time, where an
// allocation could fail in the middle of a run.  Such callers own the matrix,
// right-hand side and solution buffers and pass them in; the Krylov work
// vectors, per-block partial sums, the barrier words and the result live in
// one file-scope static device array of fixed size.
//
// Limits and rules:
//   - n <= CFD_NOALLOC_MAX_N (524288 rows, a 80^3 pressure grid); larger
//     systems are rejected with CFD_E_BADARG and a message.
//   - every GPU that loads this library holds the array (16.1 MiB) until the
//     process exits;
//   - the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress, once per device, with that device current); make
//     that first call before any stream capture;
//   - all calls share the array and it keeps the last call's contents; the
//     barrier words and the error flag are cleared on every call, the work
//     vectors are fully rewritten before use.  Calls that overlap on the GPU
//     (two streams, or two host threads) race on the array and must not be
//     issued.
// The algorithm is the solver's FP64 Jacobi-PCG: x0 = 0, stop when
// ||r||_2 <= rtol ||b||_2, one persistent cooperative kernel with bounded
// grid barriers.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../../include/cfdfs.h"
#include "common.cuh"

namespace cfd {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxN = CFD_NOALLOC_MAX_N;
constexpr int kMaxBlocks = 2048;
constexpr int kMaxDevices = 64;
// layout of the scratch array (bytes)
constexpr size_t kVecBytes = (size_t)kMaxN * sizeof(double);
constexpr size_t kOffR = 0, kOffZ = kVecBytes, kOffP = 2 * kVecBytes, kOffQ = 3 * kVecBytes;
constexpr size_t kOffPart = 4 * kVecBytes;                                    // 6 x kMaxBlocks doubles
constexpr size_t kOffCtl = kOffPart + 6 * (size_t)kMaxBlocks * sizeof(double);  // barrier[2], err, pad
constexpr size_t kOffRes = kOffCtl + 256;                                       // 4 doubles
constexpr size_t kScratchBytes = kOffRes + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

template <int NV>
__device__ __forceinline__ bool reduce_all(double (&v)[NV], double* part, int phase, unsigned* bar, int* err) {
  __shared__ double res[NV];
  const int G = gridDim.x;
  double* buf = part + (size_t)(phase & 1) * 3 * G;
  block_sum<NV>(v);
  if (threadIdx.x == 0)
    for (int k = 0; k < NV; k++) buf[(size_t)k * G + blockIdx.x] = v[k];
  if (!grid_barrier(bar, err, 2000000000ULL)) return false;
  if (threadIdx.x < 32) {
    for (int k = 0; k < NV; k++) {
      double s = 0;
      for (int i = threadIdx.x; i < G; i += 32) s += __ldcg(buf + (size_t)k * G + i);
      s = warp_sum(s);
      if (threadIdx.x == 0) res[k] = s;
    }
  }
  __syncthreads();
  for (int k = 0; k < NV; k++) v[k] = res[k];
  __syncthreads();
  return true;
}

__global__ void __launch_bounds__(kThreads) k_pcg_noalloc(int n, const int* __restrict__ rp,
                                                           const int* __restrict__ col,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ dinv,
                                                           const double* __restrict__ b, double* x, double rtol,
                                                           int maxit, unsigned char* scratch) {
  double* r = reinterpret_cast<double*>(scratch + kOffR);
  double* z = reinterpret_cast<double*>(scratch + kOffZ);
  double* p = reinterpret_cast<double*>(scratch + kOffP);
  double* q = reinterpret_cast<double*>(scratch + kOffQ);
  double* part = reinterpret_cast<double*>(scratch + kOffPart);
  unsigned* bar = reinterpret_cast<unsigned*>(scratch + kOffCtl);
  int* err = reinterpret_cast<int*>(scratch + kOffCtl + 8);
  double* result = reinterpret_cast<double*>(scratch + kOffRes);
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const long long gw = (long long)blockIdx.x * wpb + (threadIdx.x >> 5), nw = (long long)gridDim.x * wpb;
  const int r0 = (int)(n * gw / nw), r1 = (int)(n * (gw + 1) / nw);
  int phase = 0;
  double v3[3] = {0, 0, 0};
  for (int i = r0 + lane; i < r1; i += 32) {
    double bi = b[i], zi = bi * dinv[i];
    x[i] = 0.0;
    r[i] = bi;
    z[i] = zi;
    p[i] = zi;
    v3[0] += bi * bi;
    v3[1] += bi * zi;
    v3[2] += bi * bi;
  }
  bool alive = reduce_all<3>(v3, part, phase++, bar, err);
  const double bnorm = sqrt(v3[0]);
  double rz = v3[1], rn = sqrt(v3[2]);
  const double tol = rtol * bnorm;
  int its = 0, status = 1;
  if (!alive) {
    status = 3;
  } else if (!isfinite(bnorm)) {
    status = 2;
  } else if (bnorm == 0.0 || rn <= tol) {
    status = 0;
  } else {
    while (its < maxit) {
      double pq = 0;
      for (int i = r0; i < r1; i++) {
        double s = 0;
        for (int j = __ldg(rp + i) + lane; j < __ldg(rp + i + 1); j += 32) s += __ldg(val + j) * __ldcg(p + __ldg(col + j));
        s = warp_sum(s);
        if (lane == 0) {
          q[i] = s;
          pq += p[i] * s;
        }
      }
      double v1[1] = {pq};
      if (!reduce_all<1>(v1, part, phase++, bar, err)) { status = 3; break; }
      const double alpha = rz / v1[0];
      double v2[2] = {0, 0};
      for (int i = r0 + lane; i < r1; i += 32) {
        x[i] += alpha * p[i];
        double ri = r[i] - alpha * __ldcg(q + i);
        double zi = ri * dinv[i];
        r[i] = ri;
        z[i] = zi;
        v2[0] += ri * ri;
        v2[1] += ri * zi;
      }
      if (!reduce_all<2>(v2, part, phase++, bar, err)) { status = 3; break; }
      its++;
      rn = sqrt(v2[0]);
      if (!isfinite(rn)) { status = 2; break; }
      if (rn <= tol) { status = 0; break; }
      const double beta = v2[1] / rz;
      rz = v2[1];
      for (int i = r0 + lane; i < r1; i += 32) p[i] = z[i] + beta * p[i];
      if (!grid_barrier(bar, err, 2000000000ULL)) { status = 3; break; }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    result[0] = its;
    result[1] = bnorm > 0 ? rn / bnorm : 0.0;
    result[2] = status;
    result[3] = bnorm;
  }
}

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

void put_err(char* buf, int len, const char* msg) {
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", msg);
}

}  // namespace
}  // namespace cfd

extern "C" int cfd_pcg_solve_noalloc(const int* rowptr, const int* col, const double* val, const double* dinv,
                                     const double* b, double* x, int n, double rtol, int maxit, void* stream,
                                     double* info, char* errbuf, int errlen) {
  using namespace cfd;
  char msg[256];
  if (n <= 0 || n > kMaxN) {
    std::snprintf(msg, sizeof(msg), "cfd_pcg_solve_noalloc: n = %d is outside 1..%d (the size of its static work array)",
                  n, kMaxN);
    put_err(errbuf, errlen, msg);
    return CFD_E_BADARG;
  }
  if (!rowptr || !col || !val || !dinv || !b || !x || !(rtol > 0) || maxit <= 0) {
    put_err(errbuf, errlen, "cfd_pcg_solve_noalloc: null pointer, rtol <= 0 or maxit <= 0");
    return CFD_E_BADARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    put_err(errbuf, errlen, "cfd_pcg_solve_noalloc: no current CUDA device");
    return CFD_E_CUDA;
  }
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        std::snprintf(msg, sizeof(msg), "cfd_pcg_solve_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        put_err(errbuf, errlen, msg);
        return CFD_E_CUDA;
      }
      g_scratch_addr[dev] = p;
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  int sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_noalloc, kThreads, 0) != cudaSuccess ||
      per_sm < 1) {
    put_err(errbuf, errlen, "cfd_pcg_solve_noalloc: occupancy query failed");
    return CFD_E_CUDA;
  }
  long long grid = (long long)sms * per_sm;
  long long want = ((long long)n + (kThreads / 32) * 8 - 1) / ((kThreads / 32) * 8);
  if (grid > want) grid = want;
  if (grid > kMaxBlocks) grid = kMaxBlocks;
  if (grid < 1) grid = 1;
  unsigned char* base = static_cast<unsigned char*>(scratch);
  e = cudaMemsetAsync(base + kOffCtl, 0, 256, s);  // barrier words and error flag start at zero
  if (e == cudaSuccess) {
    int nn = n, mi = maxit;
    double rt = rtol;
    unsigned char* sp = base;
    void* params[] = {&nn, (void*)&rowptr, (void*)&col, (void*)&val, (void*)&dinv, (void*)&b, (void*)&x, &rt, &mi, &sp};
    e = cudaLaunchCooperativeKernel((const void*)k_pcg_noalloc, dim3((unsigned)grid), dim3(kThreads), params, 0, s);
  }
  double res[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(res, base + kOffRes, sizeof(res), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    std::snprintf(msg, sizeof(msg), "cfd_pcg_solve_noalloc: %s", cudaGetErrorString(e));
    put_err(errbuf, errlen, msg);
    return CFD_E_CUDA;
  }
  if (info) {
    info[0] = res[0];
    info[1] = res[1];
    info[2] = res[2];
  }
  switch ((int)res[2]) {
    case 0: return CFD_OK;
    case 1: put_err(errbuf, errlen, "cfd_pcg_solve_noalloc: iteration limit reached"); return CFD_E_NOCONV;
    case 2: put_err(errbuf, errlen, "cfd_pcg_solve_noalloc: non-finite residual"); return CFD_E_NONFINITE;
    default: put_err(errbuf, errlen, "cfd_pcg_solve_noalloc: bounded grid barrier timed out"); return CFD_E_TIMEOUT;
  }
}
