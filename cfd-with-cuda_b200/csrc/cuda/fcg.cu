// Flexible CG (Notay's FCG(1): each new direction is A-orthogonalised
// against the previous one, so a preconditioner that changes from one
// iteration to the next -- the U-Net -- is allowed) on the SELL-32 pressure
// matrix Z.  One iteration is
//
//   z = B(r)                                  (U-Net, launched by the host)
//   w = Z z; partial dots (z,w) (z,q) (z,r) (p,r)        k_fcg_spmv
//   beta = (z,q)/(p,q)_old, (p,q) = (z,w) - beta (z,q),
//   alpha = ((z,r) - beta (p,r)) / (p,q)                  k_fcg_coef
//   p = z - beta p, q = w - beta q, x += alpha p, r -= alpha q   k_fcg_update
//   rr = (r,r); convergence / iteration-limit / stall tests        k_fcg_check
//
// using q = Z p = Z z - beta Z p_old and (p_old, Z z) = (q_old, z).  All dots
// are FP64 with a fixed summation order (block partials, then one block).
// The state words live in device memory, and every kernel returns at once
// when the done flag is set, so the host can queue several iterations
// between status reads.
#include "common.cuh"
#include "kernels.h"

namespace cfd {

namespace {

constexpr int kFcgThreads = 256;

template <class VT>
__device__ __forceinline__ VT sell_row(const int* __restrict__ off, const int* __restrict__ col,
                                       const VT* __restrict__ val, const VT* __restrict__ x, int i) {
  const int s = i >> 5, l = i & 31;
  const int bb = __ldg(off + s) + l, w = (__ldg(off + s + 1) - __ldg(off + s)) >> 5;
  VT q = 0;
#pragma unroll 4
  for (int j = 0; j < w; j++) q += __ldcs(val + bb + 32 * j) * __ldg(x + __ldcs(col + bb + 32 * j));
  return q;
}

// r = b - Z x (warm) or r = b, x = 0; p = q = 0; partials {(b,b), (r,r)}.
template <class VT>
__global__ void __launch_bounds__(kFcgThreads) k_fcg_start(FcgArgs<VT> a, int warm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0, 0};
  if (i < a.n) {
    const VT bi = a.b[i];
    VT ri = bi;
    if (warm)
      ri = bi - sell_row(a.off, a.col, a.val, a.x, i);
    else
      a.x[i] = 0;
    a.r[i] = ri;
    a.p[i] = 0;
    a.q[i] = 0;
    v[0] = (double)bi * bi;
    v[1] = (double)ri * ri;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    a.st.part[2 * blockIdx.x] = v[0];
    a.st.part[2 * blockIdx.x + 1] = v[1];
  }
}

__global__ void k_fcg_start2(FcgState st, int nblk) {
  double v[2] = {0, 0};
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    v[0] += st.part[2 * i];
    v[1] += st.part[2 * i + 1];
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    double* sc = st.sc;
    sc[kFcgBB] = v[0];
    sc[kFcgRR] = v[1];
    sc[kFcgRRMark] = v[1];
    sc[kFcgIt] = 0;
    sc[kFcgPQ] = 1;
    sc[kFcgRtol] = st.rtol;
    sc[kFcgStall2] = st.stall2;
    sc[kFcgMaxit] = st.maxit;
    sc[kFcgWindow] = st.window;
    int done = 0;
    double status = -1;
    if (!isfinite(v[0]) || !isfinite(v[1])) {
      status = 2;
      done = 1;
    } else if (v[1] <= st.rtol * st.rtol * v[0]) {
      status = 0;
      done = 1;
    }
    sc[kFcgStatus] = status;
    st.done[0] = done;
  }
}

template <class VT>
__global__ void __launch_bounds__(kFcgThreads) k_fcg_spmv(FcgArgs<VT> a) {
  if (*a.st.done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0, 0, 0, 0};
  if (i < a.n) {
    const VT wi = sell_row(a.off, a.col, a.val, a.z, i);
    a.w[i] = wi;
    const double zi = a.z[i];
    v[0] = zi * wi;
    v[1] = zi * a.q[i];
    v[2] = zi * a.r[i];
    v[3] = (double)a.p[i] * a.r[i];
  }
  block_sum<4>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 4; k++) a.st.part[4 * blockIdx.x + k] = v[k];
}

__global__ void k_fcg_coef(FcgState st, int nblk) {
  if (*st.done) return;
  double v[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < nblk; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] += st.part[4 * i + k];
  block_sum<4>(v);
  if (threadIdx.x == 0) {
    double* sc = st.sc;
    const double zw = v[0], zq = v[1], zr = v[2], pr = v[3];
    const double beta = sc[kFcgIt] > 0 ? zq / sc[kFcgPQ] : 0.0;
    const double pq = zw - beta * zq;
    const double alpha = (zr - beta * pr) / pq;
    if (!(pq > 0.0) || !isfinite(alpha) || !isfinite(beta)) {
      // breakdown: the preconditioned direction carries no descent
      sc[kFcgStatus] = isfinite(zw) ? 4 : 2;
      st.done[0] = 1;
      return;
    }
    sc[kFcgPQ] = pq;
    sc[kFcgAlpha] = alpha;
    sc[kFcgBeta] = beta;
  }
}

template <class VT>
__global__ void __launch_bounds__(kFcgThreads) k_fcg_update(FcgArgs<VT> a) {
  if (*a.st.done) return;
  const VT alpha = (VT)a.st.sc[kFcgAlpha], beta = (VT)a.st.sc[kFcgBeta];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0};
  if (i < a.n) {
    const VT pi = a.z[i] - beta * a.p[i];
    const VT qi = a.w[i] - beta * a.q[i];
    a.p[i] = pi;
    a.q[i] = qi;
    a.x[i] += alpha * pi;
    const VT ri = a.r[i] - alpha * qi;
    a.r[i] = ri;
    v[0] = (double)ri * ri;
  }
  block_sum<1>(v);
  if (threadIdx.x == 0) a.st.part[blockIdx.x] = v[0];
}

__global__ void k_fcg_check(FcgState st, int nblk) {
  if (*st.done) return;
  double v[1] = {0};
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) v[0] += st.part[i];
  block_sum<1>(v);
  if (threadIdx.x == 0) {
    double* sc = st.sc;
    const double rr = v[0];
    const double it = sc[kFcgIt] + 1;
    const double rtol = sc[kFcgRtol], window = sc[kFcgWindow];
    sc[kFcgIt] = it;
    sc[kFcgRR] = rr;
    const bool mark = window > 0 && fmod(it, window) == 0.0;
    int done = 1;
    if (!isfinite(rr))
      sc[kFcgStatus] = 2;
    else if (rr <= rtol * rtol * sc[kFcgBB])
      sc[kFcgStatus] = 0;
    else if (it >= sc[kFcgMaxit])
      sc[kFcgStatus] = 1;
    else if (mark && rr > sc[kFcgStall2] * sc[kFcgRRMark])
      sc[kFcgStatus] = 4;
    else
      done = 0;
    if (!done && mark) sc[kFcgRRMark] = rr;
    st.done[0] = done;
  }
}

int nblocks(int n) { return (n + kFcgThreads - 1) / kFcgThreads; }

}  // namespace

int fcg_blocks(int n) { return nblocks(n); }

template <class VT>
cudaError_t launch_fcg_start(const FcgArgs<VT>& a, int warm, cudaStream_t s) {
  const int g = nblocks(a.n);
  k_fcg_start<VT><<<g, kFcgThreads, 0, s>>>(a, warm);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_fcg_start2<<<1, 1024, 0, s>>>(a.st, g);
  return cudaGetLastError();
}

template <class VT>
cudaError_t launch_fcg_spmv(const FcgArgs<VT>& a, cudaStream_t s) {
  const int g = nblocks(a.n);
  k_fcg_spmv<VT><<<g, kFcgThreads, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_fcg_coef<<<1, 1024, 0, s>>>(a.st, g);
  return cudaGetLastError();
}

template <class VT>
cudaError_t launch_fcg_update(const FcgArgs<VT>& a, cudaStream_t s) {
  const int g = nblocks(a.n);
  k_fcg_update<VT><<<g, kFcgThreads, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_fcg_check<<<1, 1024, 0, s>>>(a.st, g);
  return cudaGetLastError();
}

template cudaError_t launch_fcg_start<float>(const FcgArgs<float>&, int, cudaStream_t);
template cudaError_t launch_fcg_start<double>(const FcgArgs<double>&, int, cudaStream_t);
template cudaError_t launch_fcg_spmv<float>(const FcgArgs<float>&, cudaStream_t);
template cudaError_t launch_fcg_spmv<double>(const FcgArgs<double>&, cudaStream_t);
template cudaError_t launch_fcg_update<float>(const FcgArgs<float>&, cudaStream_t);
template cudaError_t launch_fcg_update<double>(const FcgArgs<double>&, cudaStream_t);

}  // namespace cfd
