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
#include <algorithm>

#include "common.cuh"
#include "fcg_common.cuh"
#include "kernels.h"
#include "sell_stream.cuh"

namespace cfd {

namespace {

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

// Block sums of the SpMV's partials; the last block to finish forms the
// coefficients beta_j, (p,q) and alpha of the iteration.
template <int MD, class VT>
__device__ __forceinline__ void fcg_spmv_finish(const FcgArgs<VT>& a, double (&v)[fcg_parts<MD>()], int nd, int m,
                                                int it) {
  constexpr int NV = fcg_parts<MD>();
  block_sum<NV>(v);
  if (!post_partials<NV>(v, a.st.part, a.st.cnt)) return;
  gather_partials<NV>(a.st.part, gridDim.x, v);
  if (threadIdx.x == 0) {
    double* s = a.st.sc;
    if (ld_volatile_i32(a.st.err)) {
      s[kFcgStatus] = 3;  // a bounded wait of the matrix stream gave up
      a.st.done[0] = 1;
      return;
    }
    double pq = v[0], pr = v[1];
    double beta[kFcgMaxM];
#pragma unroll
    for (int j = 0; j < kFcgMaxM; j++) {
      beta[j] = 0.0;
      if (j < MD && j < nd) {
        beta[j] = v[2 + j] / s[kFcgPQ0 + j];
        pq -= beta[j] * v[2 + j];
        pr -= beta[j] * v[2 + MD + j];
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
    // the new direction takes the oldest (or, anchored, the last) slot
    s[kFcgPQ0 + fcg_slot(it, m, (int)s[kFcgAnchor])] = pq;
  }
}

// r = b - Z x (warm) or r = b, x = 0; partials {(b,b), (r,r)}; the last
// block initialises the state words.
template <class VT>
__global__ void __launch_bounds__(kFcgThreads) k_fcg_start(FcgArgs<VT> a, int warm) {
  pdl_wait();
  pdl_trigger();
  double v[2] = {0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const VT bi = a.b[i];
    VT ri = bi;
    if (warm)
      ri = bi - sell_row(a.off, a.col, a.val, a.x, i);
    else
      a.x[i] = 0;
    a.r[i] = ri;
    if (a.z1) a.z1[i] = a.dinv[i] * ri;
    v[0] += (double)bi * bi;
    v[1] += (double)ri * ri;
  }
  block_sum<2>(v);
  if (!post_partials<2>(v, a.st.part, a.st.cnt)) return;
  gather_partials<2>(a.st.part, gridDim.x, v);
  if (threadIdx.x == 0) {
    const FcgState& st = a.st;
    double* sc = st.sc;
    *st.err = 0;
    sc[kFcgBB] = v[0];
    sc[kFcgRR] = v[1];
    sc[kFcgRRMark] = v[1];
    sc[kFcgIt] = 0;
    sc[kFcgRtol] = st.rtol;
    sc[kFcgStall2] = st.stall2;
    sc[kFcgMaxit] = st.maxit;
    sc[kFcgWindow] = st.window;
    sc[kFcgM] = st.m;
    sc[kFcgAnchor] = st.anchor;
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

// w = Z z with the matrix streamed through shared memory (ChunkStream, as in
// the persistent PCG): 16 warps per block, each owning a contiguous range of
// 32-row slices, lane = row.
template <class VT, int MD>
__global__ void __launch_bounds__(kPcgThreads, 2) k_fcg_spmv(FcgArgs<VT> a) {
  pdl_wait();
  pdl_trigger();
  if (*a.st.done) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const double* sc = a.st.sc;
  const int m = (int)sc[kFcgM], it = (int)sc[kFcgIt];
  const int nd = it < m ? it : m;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nslices = (a.n + 31) >> 5;
  const int W = gridDim.x * kPcgWarps, gw = blockIdx.x * kPcgWarps + wib;
  Chunk<VT>* chunks = reinterpret_cast<Chunk<VT>*>(smem);
  unsigned long long* mbars =
      reinterpret_cast<unsigned long long*>(smem + (size_t)kPcgWarps * kNbuf<VT> * sizeof(Chunk<VT>));
  ChunkStream<VT> st;
  st.off = a.off;
  st.col = a.col;
  st.val = a.val;
  st.buf = chunks + wib * kNbuf<VT>;
  st.mbar = mbars + wib * kNbuf<VT>;
  st.s_begin = (int)((long long)nslices * gw / W);
  st.s_end = (int)((long long)nslices * (gw + 1) / W);
  st.is = st.cs = st.s_begin;
  st.ik = st.ck = 0;
  st.nbi = st.nbc = 0;
  st.parity = 0;
  st.failed = false;
  if (lane == 0)
    for (int k = 0; k < kNbuf<VT>; k++) mbar_init(st.mbar + k, 1);
  mbar_init_fence();
  __syncwarp();
  st.start(lane);
  double v[fcg_parts<MD>()];
#pragma unroll
  for (int k = 0; k < fcg_parts<MD>(); k++) v[k] = 0.0;
  for (int sl = st.s_begin; sl < st.s_end; sl++) {
    VT acc = 0;
    const int wd = (__ldg(a.off + sl + 1) - __ldg(a.off + sl)) >> 5;
    for (int c0 = 0; c0 < wd; c0 += kCh) {
      if (st.wait(a.st.err, a.st.timeout_ns)) acc += chunk_dot<VT>(st.buf + st.nbc, min(kCh, wd - c0), lane, a.z);
      st.release(lane);
    }
    const int i = sl * 32 + lane;
    if (i < a.n) fcg_row_dots<MD>(a, i, a.z[i], acc, nd, v);
  }
  if (!st.failed) st.drain(a.st.timeout_ns);
  fcg_spmv_finish<MD>(a, v, nd, m, it);
}

// DOTS = false: w = Z z only (the Jacobi part of the split iteration).
template <class VT, int MD, bool DOTS>
__global__ void __launch_bounds__(kPcgThreads, 2) k_fcg_spmv_stencil(FcgArgs<VT> a) {
  pdl_wait();
  pdl_trigger();
  if (*a.st.done) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const double* sc = a.st.sc;
  const int m = (int)sc[kFcgM], it = (int)sc[kFcgIt];
  const int nd = it < m ? it : m;
  const int n = a.n, fx = a.fd[0], fxy = a.fd[0] * a.fd[1];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nslices = (n + 31) >> 5;
  const int W = gridDim.x * kPcgWarps, gw = blockIdx.x * kPcgWarps + wib;
  const int s0 = (int)((long long)nslices * gw / W), s1 = (int)((long long)nslices * (gw + 1) / W);
  constexpr unsigned kChunkBytes = kStTaps * 32 * sizeof(VT);
  VT* buf = reinterpret_cast<VT*>(smem) + (size_t)wib * kStBuf * kStTaps * 32;
  unsigned long long* mbar =
      reinterpret_cast<unsigned long long*>(smem + (size_t)kPcgWarps * kStBuf * kChunkBytes) + wib * kStBuf;
  const int total = (s1 - s0) * 5;  // chunks of this warp
  if (lane == 0)
    for (int b = 0; b < kStBuf; b++) mbar_init(mbar + b, 1);
  mbar_init_fence();
  __syncwarp();
  // the coefficients are read once per iteration: evict-first in L2, so the
  // vectors and the coarse inverse stay
  const unsigned long long once = l2_evict_first();
  auto issue = [&](int k) {  // chunk k of the warp's range into buffer k % kStBuf
    if (lane == 0 && k < total) {
      const int b = k % kStBuf;
      const VT* src = a.stencil + ((size_t)(s0 + k / 5) * 125 + (k % 5) * kStTaps) * 32;
      fence_proxy_async_smem();
      mbar_expect_tx(mbar + b, kChunkBytes);
      bulk_g2s_hint(buf + (size_t)b * kStTaps * 32, src, kChunkBytes, mbar + b, once);
    }
  };
  for (int k = 0; k < kStBuf; k++) issue(k);
  bool ok = true;
  int kfail = 0;
  const VT* __restrict__ z = a.z;
  const int reach = 2 + 2 * fx + 2 * fxy;  // largest |j - i| of a tap
  double v[fcg_parts<MD>()];
#pragma unroll
  for (int k = 0; k < fcg_parts<MD>(); k++) v[k] = 0.0;
  int k = 0;
  for (int sl = s0; sl < s1; sl++) {
    const int i = sl * 32 + lane;
    const bool inside = sl * 32 >= reach && sl * 32 + 31 + reach < n;  // warp-uniform
    VT acc[5] = {0, 0, 0, 0, 0};
    for (int dz = -2; dz <= 2; dz++, k++) {
      const int b = k % kStBuf;
      // the gathers below shuffle across the warp: every lane takes the
      // same branch, so the outcome of the wait is made warp-uniform
      if (ok && !__all_sync(0xffffffffu, mbar_wait_bounded(mbar + b, (unsigned)((k / kStBuf) & 1),
                                                           a.st.timeout_ns))) {
        ok = false;
        kfail = k;
        if (lane == 0) atomicExch(a.st.err, 1);
      }
      if (ok) {
        const VT* q = buf + (size_t)b * kStTaps * 32 + lane;
        if (inside)
          stencil_plane_shfl<false, true>(q, z, i + fxy * dz, fx, n, lane, acc);
        else
          stencil_plane_shfl<true, true>(q, z, i + fxy * dz, fx, n, lane, acc);
      }
      __syncwarp();
      if (ok) issue(k + kStBuf);
    }
    if (i < n) {
      const VT wi = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + acc[4];
      if constexpr (DOTS)
        fcg_row_dots<MD>(a, i, z[i], wi, nd, v);
      else
        a.w[i] = wi;
    }
  }
  if (!ok && lane == 0) {
    // a bounded wait gave up: give the copies still in flight one more
    // bounded wait before the block (and its shared memory) ends
    for (int kk = kfail; kk < kfail + kStBuf && kk < total; kk++)
      mbar_wait_bounded(mbar + kk % kStBuf, (unsigned)((kk / kStBuf) & 1), a.st.timeout_ns);
  }
  if constexpr (DOTS) fcg_spmv_finish<MD>(a, v, nd, m, it);
}

// The second half of the split iteration: z = z1 + P e (trilinear
// prolongation of the coarse solution), w = w + (Z P) e with the 27 taps of
// the row's coarse box, the dot products of the iteration, and in the last
// block the coefficients (as the SpMV kernels do).  Identity numbering.
constexpr int kCombineThreads = 256;
template <class VT, int MD>
__global__ void __launch_bounds__(kCombineThreads) k_fcg_combine(FcgArgs<VT> a, CoarseArgs<VT> ca,
                                                                 const float* __restrict__ wst,
                                                                 const int* __restrict__ wlo,
                                                                 const VT* __restrict__ e) {
  pdl_wait();
  pdl_trigger();
  if (*a.st.done) return;
  const double* sc = a.st.sc;
  const int m = (int)sc[kFcgM], it = (int)sc[kFcgIt];
  const int nd = it < m ? it : m;
  const int fx = ca.fd[0], fy = ca.fd[1];
  const int cx = ca.cd[0], cxy = ca.cd[0] * ca.cd[1];
  const int bx = ca.cd[0] > 1, by = ca.cd[1] > 1, bz = ca.cd[2] > 1;
  double v[fcg_parts<MD>()];
#pragma unroll
  for (int k = 0; k < fcg_parts<MD>(); k++) v[k] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const int x = i % fx, y = (i / fx) % fy, zz = i / (fx * fy);
    const int ix = ca.i0x[x], iy = ca.i0y[y], iz = ca.i0z[zz];
    const VT wx = (VT)ca.fx[x], wy = (VT)ca.fy[y], wz = (VT)ca.fz[zz];
    const VT* e0 = e + ix + cx * iy + cxy * iz;
    VT pe = 0;
#pragma unroll
    for (int cnr = 0; cnr < 8; cnr++) {
      const int dx = cnr & 1, dy = (cnr >> 1) & 1, dz = cnr >> 2;
      if ((dx && !bx) || (dy && !by) || (dz && !bz)) continue;
      const VT wt = (dx ? wx : 1 - wx) * (dy ? wy : 1 - wy) * (dz ? wz : 1 - wz);
      pe += wt * e0[dx + cx * dy + cxy * dz];
    }
    const VT zi = a.z1[i] + pe;
    a.z[i] = zi;
    const float* wr = wst + (size_t)(i >> 5) * 27 * 32 + (i & 31);
    const VT* eb = e + wlo[i];
    VT we = 0;
#pragma unroll
    for (int t = 0; t < 27; t++) {
      const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
      we += (VT)__ldcs(wr + t * 32) * eb[dx + cx * dy + cxy * dz];
    }
    fcg_row_dots<MD>(a, i, zi, a.w[i] + we, nd, v);
  }
  fcg_spmv_finish<MD>(a, v, nd, m, it);
}

template <class VT>
__global__ void __launch_bounds__(kFcgThreads) k_fcg_update(FcgArgs<VT> a) {
  pdl_wait();
  pdl_trigger();
  if (*a.st.done) return;
  const double* sc = a.st.sc;
  const int m = (int)sc[kFcgM], it = (int)sc[kFcgIt];
  const int nd = it < m ? it : m, slot = fcg_slot(it, m, (int)sc[kFcgAnchor]);
  const VT alpha = (VT)sc[kFcgAlpha];
  VT beta[kFcgMaxM];
#pragma unroll
  for (int j = 0; j < kFcgMaxM; j++) beta[j] = (VT)sc[kFcgBeta0 + j];
  const size_t n = (size_t)a.n;
  double v[1] = {0};
  // UPD grid-stride elements per thread with all their loads issued before
  // any store (the element order, and so the order of the (r, r) sum, is the
  // grid-stride order)
  constexpr int UPD = 4;
  const int stride = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += UPD * stride) {
    VT pi[UPD], qi[UPD], xo[UPD], ro[UPD];
#pragma unroll
    for (int u = 0; u < UPD; u++) {
      const int i = i0 + u * stride;
      if (i < a.n) {
        pi[u] = a.z[i];
        qi[u] = a.w[i];
        xo[u] = a.x[i];
        ro[u] = a.r[i];
#pragma unroll
        for (int j = 0; j < kFcgMaxM; j++) {
          if (j < nd) {
            pi[u] -= beta[j] * a.p[j * n + i];
            qi[u] -= beta[j] * a.q[j * n + i];
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < UPD; u++) {
      const int i = i0 + u * stride;
      if (i < a.n) {
        a.p[slot * n + i] = pi[u];
        a.q[slot * n + i] = qi[u];
        a.x[i] = xo[u] + alpha * pi[u];
        const VT ri = ro[u] - alpha * qi[u];
        a.r[i] = ri;
        if (a.z1) a.z1[i] = a.dinv[i] * ri;
        v[0] += (double)ri * ri;
      }
    }
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

// coef[tap][row] of the structured form of a CSR matrix (identity numbering
// on the grid fd); *bad = 1 when a coupling reaches beyond two grid steps.
template <class VT>
__global__ void k_stencil_build(int n, Int3 fd, const int* __restrict__ rp, const int* __restrict__ col,
                                const double* __restrict__ val, VT* coef, int* bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int x = i % fd.v[0], y = (i / fd.v[0]) % fd.v[1], z = i / (fd.v[0] * fd.v[1]);
    for (int k = rp[i]; k < rp[i + 1]; k++) {
      const int j = col[k];
      const int dx = j % fd.v[0] - x, dy = (j / fd.v[0]) % fd.v[1] - y, dz = j / (fd.v[0] * fd.v[1]) - z;
      if (dx < -2 || dx > 2 || dy < -2 || dy > 2 || dz < -2 || dz > 2) {
        atomicExch(bad, 1);
        continue;
      }
      coef[((size_t)(i >> 5) * 125 + (dz + 2) * 25 + (dy + 2) * 5 + (dx + 2)) * 32 + (i & 31)] = (VT)val[k];
    }
  }
}

int nblocks(int n) {
  const int g = (n + kFcgThreads - 1) / kFcgThreads;
  return g < kFcgMaxBlocks ? g : kFcgMaxBlocks;
}

}  // namespace

int fcg_blocks(int n) { return nblocks(n); }
size_t stencil_elems(int n) { return (size_t)((n + 31) >> 5) * 125 * 32; }
size_t zp_elems(int n) { return (size_t)((n + 31) >> 5) * 27 * 32; }
int fcg_part_words(int n) { return kFcgParts * (nblocks(n) > kFcgMaxBlocks ? nblocks(n) : kFcgMaxBlocks); }

template <class VT>
cudaError_t launch_fcg_start(const FcgArgs<VT>& a, int warm, cudaStream_t s) {
  if (a.st.m < 1 || a.st.m > kFcgMaxM) return cudaErrorInvalidValue;
  if (a.st.anchor < 0 || (a.st.anchor > 0 && a.st.m != a.st.anchor + 1)) return cudaErrorInvalidValue;
  return launch_k(a.pdl != 0, k_fcg_start<VT>, dim3(nblocks(a.n)), dim3(kFcgThreads), 0, s, a, warm);
}

template <class VT, int MD, bool DOTS>
cudaError_t launch_stencil_kernel(const FcgArgs<VT>& a, cudaStream_t s) {
  // one wave of two blocks of 16 warps per SM
  const size_t smem = stencil_smem_bytes<VT>();
  cudaError_t e = cudaFuncSetAttribute(k_fcg_spmv_stencil<VT, MD, DOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  return launch_k(a.pdl != 0, k_fcg_spmv_stencil<VT, MD, DOTS>, dim3(a.spmv_grid), dim3(kPcgThreads), smem, s, a);
}

template <class VT, int MD>
cudaError_t launch_fcg_spmv_md(const FcgArgs<VT>& a, cudaStream_t s) {
  if (a.stencil) return launch_stencil_kernel<VT, MD, true>(a, s);
  const size_t smem = pcg_smem_bytes<VT>();
  cudaError_t e = cudaFuncSetAttribute(k_fcg_spmv<VT, MD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return launch_k(a.pdl != 0, k_fcg_spmv<VT, MD>, dim3(a.spmv_grid), dim3(kPcgThreads), smem, s, a);
}

// the SpMV's dot partials are sized for the solve's window m: 1 (CG with a
// fixed preconditioner), 2 (one anchored direction and the last), up to 4,
// up to kFcgMaxM
template <class VT>
cudaError_t launch_fcg_spmv(const FcgArgs<VT>& a, cudaStream_t s) {
  if (a.spmv_grid < 1 || a.spmv_grid > kFcgMaxBlocks) return cudaErrorInvalidValue;
  if (a.st.m < 1 || a.st.m > kFcgMaxM) return cudaErrorInvalidValue;
  if (a.st.m == 1) return launch_fcg_spmv_md<VT, 1>(a, s);
  if (a.st.m == 2) return launch_fcg_spmv_md<VT, 2>(a, s);
  if (a.st.m <= 4) return launch_fcg_spmv_md<VT, 4>(a, s);
  return launch_fcg_spmv_md<VT, kFcgMaxM>(a, s);
}

template <class VT>
cudaError_t launch_fcg_spmv_jacobi(const FcgArgs<VT>& a, cudaStream_t s) {
  if (!a.stencil || !a.z1 || a.spmv_grid < 1 || a.spmv_grid > kFcgMaxBlocks) return cudaErrorInvalidValue;
  FcgArgs<VT> b = a;
  b.z = a.z1;  // w = Z z1
  return launch_stencil_kernel<VT, 1, false>(b, s);
}

template <class VT, int MD>
cudaError_t launch_combine_md(const FcgArgs<VT>& a, const CoarseArgs<VT>& ca, const float* wst, const int* wlo,
                              const VT* e, cudaStream_t s) {
  return launch_k(a.pdl != 0, k_fcg_combine<VT, MD>, dim3(nblocks(a.n)), dim3(kCombineThreads), 0, s, a, ca, wst,
                  wlo, e);
}

template <class VT>
cudaError_t launch_fcg_combine(const FcgArgs<VT>& a, const CoarseArgs<VT>& ca, const float* wst, const int* wlo,
                               const VT* e, cudaStream_t s) {
  if (!a.z1 || ca.pmap || a.st.m < 1 || a.st.m > kFcgMaxM) return cudaErrorInvalidValue;
  if ((long long)ca.fd[0] * ca.fd[1] * ca.fd[2] != a.n) return cudaErrorInvalidValue;
  if (a.st.m == 1) return launch_combine_md<VT, 1>(a, ca, wst, wlo, e, s);
  if (a.st.m <= 4) return launch_combine_md<VT, 4>(a, ca, wst, wlo, e, s);
  return launch_combine_md<VT, kFcgMaxM>(a, ca, wst, wlo, e, s);
}

template <class VT>
cudaError_t launch_fcg_update(const FcgArgs<VT>& a, cudaStream_t s) {
  int grid = nblocks(a.n);
  if (a.upd_grid > 0 && a.upd_grid < grid) grid = a.upd_grid;
  return launch_k(a.pdl != 0, k_fcg_update<VT>, dim3(grid), dim3(kFcgThreads), 0, s, a);
}

template <class VT>
cudaError_t launch_stencil_build(int n, const int fd[3], const int* rp, const int* col, const double* val, VT* coef,
                                 int* bad, cudaStream_t s) {
  Int3 g;
  for (int k = 0; k < 3; k++) g.v[k] = fd[k];
  cudaError_t e = cudaMemsetAsync(coef, 0, stencil_elems(n) * sizeof(VT), s);
  if (e != cudaSuccess) return e;
  k_stencil_build<VT><<<(n + 255) / 256, 256, 0, s>>>(n, g, rp, col, val, coef, bad);
  return cudaGetLastError();
}

template cudaError_t launch_stencil_build<float>(int, const int*, const int*, const int*, const double*, float*, int*,
                                                 cudaStream_t);
template cudaError_t launch_fcg_start<float>(const FcgArgs<float>&, int, cudaStream_t);
template cudaError_t launch_fcg_start<double>(const FcgArgs<double>&, int, cudaStream_t);
template cudaError_t launch_fcg_spmv<float>(const FcgArgs<float>&, cudaStream_t);
template cudaError_t launch_fcg_spmv<double>(const FcgArgs<double>&, cudaStream_t);
template cudaError_t launch_fcg_update<float>(const FcgArgs<float>&, cudaStream_t);
template cudaError_t launch_fcg_update<double>(const FcgArgs<double>&, cudaStream_t);
template cudaError_t launch_fcg_spmv_jacobi<float>(const FcgArgs<float>&, cudaStream_t);
template cudaError_t launch_fcg_combine<float>(const FcgArgs<float>&, const CoarseArgs<float>&, const float*,
                                               const int*, const float*, cudaStream_t);

}  // namespace cfd
