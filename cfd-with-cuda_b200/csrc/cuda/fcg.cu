// Truncated flexible CG, FCG(m) (Notay 2000: each new direction is
// Z-orthogonalised against the last m directions, so a preconditioner that
// changes from one iteration to the next -- the U-Net -- is allowed; m = 1
// is the classical FCG(1) / Polak-Ribiere form) on the SELL-32 pressure
// matrix Z.  One iteration is
//
//   z = B(r)                                  (U-Net, launched by the host)
//   w = Z z; partial dots (z,w) (z,r) (z,q_j) (p_j,r), j < nd      k_fcg_spmv
//     last block: beta_j = (z,q_j)/(p_j,q_j), (p,q) = (z,w) - sum beta_j (z,q_j),
//                 alpha = ((z,r) - sum beta_j (p_j,r)) / (p,q)
//   p = z - sum beta_j p_j, q = w - sum beta_j q_j  (into the ring slot of
//   the oldest direction), x += alpha p, r -= alpha q, partial (r,r)
//                                                                k_fcg_update
//     last block: convergence / iteration-limit / stall tests
//
// using q = Z p, (p_j, q_i) = 0 for i != j inside the window, and nd =
// min(iteration, m) stored directions.  All dots are FP64; the last block to
// finish sums the per-block partials in block order, so results do not
// depend on which block finishes last.  The state words live in device
// memory, and every kernel returns at once when the done flag is set, so the
// host can queue several iterations between status reads.
#include "common.cuh"
#include "kernels.h"

namespace cfd {

namespace {

constexpr int kFcgThreads = 256;
constexpr int kFcgParts = 2 + 2 * kFcgMaxM;  // partial sums per block

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

// Stores this block's NV partials, and returns true in every thread of the
// block that finished last (its thread 0 has re-armed the counter); the
// caller then sums part[] over all blocks.
template <int NV>
__device__ __forceinline__ bool post_partials(const double (&v)[NV], double* part, unsigned* cnt) {
  __shared__ int s_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) part[NV * blockIdx.x + k] = v[k];
    __threadfence();
    const unsigned prev = atomicAdd(cnt, 1u);
    s_last = prev == gridDim.x - 1;
    if (s_last) {
      atomicExch(cnt, 0u);
      __threadfence();
    }
  }
  __syncthreads();
  return s_last != 0;
}

// Sum of the NV partials of all blocks (fixed order), valid in thread 0.
template <int NV>
__device__ __forceinline__ void gather_partials(const double* part, int nblk, double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] += __ldcg(part + NV * b + k);
  block_sum<NV>(v);
}

// r = b - Z x (warm) or r = b, x = 0; partials {(b,b), (r,r)}; the last
// block initialises the state words.
template <class VT>
__global__ void __launch_bounds__(kFcgThreads) k_fcg_start(FcgArgs<VT> a, int warm) {
  double v[2] = {0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const VT bi = a.b[i];
    VT ri = bi;
    if (warm)
      ri = bi - sell_row(a.off, a.col, a.val, a.x, i);
    else
      a.x[i] = 0;
    a.r[i] = ri;
    v[0] += (double)bi * bi;
    v[1] += (double)ri * ri;
  }
  block_sum<2>(v);
  if (!post_partials<2>(v, a.st.part, a.st.cnt)) return;
  gather_partials<2>(a.st.part, gridDim.x, v);
  if (threadIdx.x == 0) {
    const FcgState& st = a.st;
    double* sc = st.sc;
    sc[kFcgBB] = v[0];
    sc[kFcgRR] = v[1];
    sc[kFcgRRMark] = v[1];
    sc[kFcgIt] = 0;
    sc[kFcgRtol] = st.rtol;
    sc[kFcgStall2] = st.stall2;
    sc[kFcgMaxit] = st.maxit;
    sc[kFcgWindow] = st.window;
    sc[kFcgM] = st.m;
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
  const double* sc = a.st.sc;
  const int m = (int)sc[kFcgM], it = (int)sc[kFcgIt];
  const int nd = it < m ? it : m;
  const size_t n = (size_t)a.n;
  double v[kFcgParts];
#pragma unroll
  for (int k = 0; k < kFcgParts; k++) v[k] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const VT wi = sell_row(a.off, a.col, a.val, a.z, i);
    a.w[i] = wi;
    const double zi = a.z[i], ri = a.r[i];
    v[0] += zi * wi;
    v[1] += zi * ri;
#pragma unroll
    for (int j = 0; j < kFcgMaxM; j++) {
      if (j < nd) {
        v[2 + j] += zi * (double)a.q[j * n + i];
        v[2 + kFcgMaxM + j] += (double)a.p[j * n + i] * ri;
      }
    }
  }
  block_sum<kFcgParts>(v);
  if (!post_partials<kFcgParts>(v, a.st.part, a.st.cnt)) return;
  gather_partials<kFcgParts>(a.st.part, gridDim.x, v);
  if (threadIdx.x == 0) {
    double* s = a.st.sc;
    double pq = v[0], pr = v[1];
    double beta[kFcgMaxM];
#pragma unroll
    for (int j = 0; j < kFcgMaxM; j++) {
      beta[j] = 0.0;
      if (j < nd) {
        beta[j] = v[2 + j] / s[kFcgPQ0 + j];
        pq -= beta[j] * v[2 + j];
        pr -= beta[j] * v[2 + kFcgMaxM + j];
      }
    }
    const double alpha = pr / pq;
    bool bad = !(pq > 0.0) || !isfinite(alpha);
#pragma unroll
    for (int j = 0; j < kFcgMaxM; j++) bad = bad || !isfinite(beta[j]);
    if (bad) {
      // breakdown: the preconditioned direction carries no descent
      s[kFcgStatus] = isfinite(v[0]) ? 4 : 2;
      a.st.done[0] = 1;
      return;
    }
#pragma unroll
    for (int j = 0; j < kFcgMaxM; j++) s[kFcgBeta0 + j] = beta[j];
    s[kFcgAlpha] = alpha;
    s[kFcgPQ0 + it % m] = pq;  // the new direction takes the oldest slot
  }
}

template <class VT>
__global__ void __launch_bounds__(kFcgThreads) k_fcg_update(FcgArgs<VT> a) {
  if (*a.st.done) return;
  const double* sc = a.st.sc;
  const int m = (int)sc[kFcgM], it = (int)sc[kFcgIt];
  const int nd = it < m ? it : m, slot = it % m;
  const VT alpha = (VT)sc[kFcgAlpha];
  VT beta[kFcgMaxM];
#pragma unroll
  for (int j = 0; j < kFcgMaxM; j++) beta[j] = (VT)sc[kFcgBeta0 + j];
  const size_t n = (size_t)a.n;
  double v[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    VT pi = a.z[i], qi = a.w[i];
#pragma unroll
    for (int j = 0; j < kFcgMaxM; j++) {
      if (j < nd) {
        pi -= beta[j] * a.p[j * n + i];
        qi -= beta[j] * a.q[j * n + i];
      }
    }
    a.p[slot * n + i] = pi;
    a.q[slot * n + i] = qi;
    a.x[i] += alpha * pi;
    const VT ri = a.r[i] - alpha * qi;
    a.r[i] = ri;
    v[0] += (double)ri * ri;
  }
  block_sum<1>(v);
  if (!post_partials<1>(v, a.st.part, a.st.cnt)) return;
  gather_partials<1>(a.st.part, gridDim.x, v);
  if (threadIdx.x == 0) {
    double* s = a.st.sc;
    const double rr = v[0];
    const double itn = s[kFcgIt] + 1;
    const double rtol = s[kFcgRtol], window = s[kFcgWindow];
    s[kFcgIt] = itn;
    s[kFcgRR] = rr;
    const bool mark = window > 0 && fmod(itn, window) == 0.0;
    int done = 1;
    if (!isfinite(rr))
      s[kFcgStatus] = 2;
    else if (rr <= rtol * rtol * s[kFcgBB])
      s[kFcgStatus] = 0;
    else if (itn >= s[kFcgMaxit])
      s[kFcgStatus] = 1;
    else if (mark && rr > s[kFcgStall2] * s[kFcgRRMark])
      s[kFcgStatus] = 4;
    else
      done = 0;
    if (!done && mark) s[kFcgRRMark] = rr;
    a.st.done[0] = done;
  }
}

int nblocks(int n) {
  const int g = (n + kFcgThreads - 1) / kFcgThreads;
  return g < kFcgMaxBlocks ? g : kFcgMaxBlocks;
}

}  // namespace

int fcg_blocks(int n) { return nblocks(n); }
int fcg_part_words(int n) { return kFcgParts * nblocks(n); }

template <class VT>
cudaError_t launch_fcg_start(const FcgArgs<VT>& a, int warm, cudaStream_t s) {
  if (a.st.m < 1 || a.st.m > kFcgMaxM) return cudaErrorInvalidValue;
  k_fcg_start<VT><<<nblocks(a.n), kFcgThreads, 0, s>>>(a, warm);
  return cudaGetLastError();
}

template <class VT>
cudaError_t launch_fcg_spmv(const FcgArgs<VT>& a, cudaStream_t s) {
  k_fcg_spmv<VT><<<nblocks(a.n), kFcgThreads, 0, s>>>(a);
  return cudaGetLastError();
}

template <class VT>
cudaError_t launch_fcg_update(const FcgArgs<VT>& a, cudaStream_t s) {
  k_fcg_update<VT><<<nblocks(a.n), kFcgThreads, 0, s>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_fcg_start<float>(const FcgArgs<float>&, int, cudaStream_t);
template cudaError_t launch_fcg_start<double>(const FcgArgs<double>&, int, cudaStream_t);
template cudaError_t launch_fcg_spmv<float>(const FcgArgs<float>&, cudaStream_t);
template cudaError_t launch_fcg_spmv<double>(const FcgArgs<double>&, cudaStream_t);
template cudaError_t launch_fcg_update<float>(const FcgArgs<float>&, cudaStream_t);
template cudaError_t launch_fcg_update<double>(const FcgArgs<double>&, cudaStream_t);

}  // namespace cfd
