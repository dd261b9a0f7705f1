// Jacobi-preconditioned CG on the pressure Schur operator Z as one
// persistent cooperative kernel per solve (replaces cusp::krylov::cg with
// precond::diagonal, CUDAcodes.cu:418-451, and MKL dcg, blascoCodinaHuerta.cpp:
// 3981-4055).
//
// Z is stored SELL-32; a warp owns a contiguous range of 32-row slices and
// streams their columns and values through shared memory with bulk
// asynchronous copies (ChunkStream).  The iteration is the pipelined form of
// PCG (k_pcg below): the three dot products of an iteration are posted before
// its SpMV and collected after it, and blocks wait only for the neighbouring
// blocks whose rows they gather, so no grid-wide barrier sits on the critical
// path.  Every block sums the posted partials in the same fixed order
// (FP64), so all blocks take the same decisions.  Every wait (progress
// flag, arrival counter, mbarrier) is bounded and reports a timeout status.
// Stopping rule: ||r||_2 <= rtol ||b||_2 on the recursively updated residual.
#include <algorithm>
#include <vector>

#include "kernels.h"
#include "sell_stream.cuh"

namespace cfd {

namespace {

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) { return ld_acquire_u32(p); }
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Block-level synchronisation of the pipelined solve (all waits bounded):
//   publish(k)        this block's own rows of phase k are written
//   wait_nb(k)        every block owning a row this block gathers reached k
//   arrive/wait_red   monotonic arrival counter of the per-iteration reduction
struct BlockSync {
  unsigned* cnt;
  unsigned* prog;
  int lo, hi;
  int* err;
  unsigned long long timeout_ns;

  __device__ void publish(unsigned k) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release_gpu(prog + blockIdx.x, k);
    }
  }
  __device__ bool wait_nb(unsigned k) {
    __shared__ int ok;
    if (threadIdx.x < 32) {
      // one lane per neighbour block, all polled at once
      int good = 1;
      const unsigned long long t0 = global_ns();
      for (int j0 = lo; j0 <= hi; j0 += 32) {
        const int j = j0 + (int)threadIdx.x;
        bool done = j > hi;
        while (true) {
          if (!done) done = ld_acquire_gpu(prog + j) >= k;
          if (__all_sync(0xffffffffu, done)) break;
          // the whole warp gives up together: every lane takes the same
          // sequence of warp-wide votes
          if (__any_sync(0xffffffffu, ld_volatile_i32(err) != 0 || global_ns() - t0 > timeout_ns)) {
            good = 0;
            break;
          }
        }
        if (!good) break;
      }
      __threadfence();
      if (threadIdx.x == 0) {
        if (!good) atomicExch(err, 1);
        ok = good;
      }
    }
    __syncthreads();
    return ok != 0;
  }
  // partials already written by thread 0 of this block
  __device__ void arrive() {
    if (threadIdx.x == 0) {
      __threadfence();
      red_release_add(cnt, 1u);
    }
  }
  // Waits until `target` arrivals, then every block sums the partials in the
  // same fixed order (FP64): all blocks see identical values.
  template <int NV>
  __device__ bool wait_red(unsigned target, const double* buf, double (&v)[NV]) {
    __shared__ double res[NV];
    __shared__ int ok;
    const int G = gridDim.x;
    if (threadIdx.x < 32) {
      int good = 1;
      const unsigned long long t0 = global_ns();
      while (ld_acquire_gpu(cnt) < target) {
        if (ld_volatile_i32(err) || global_ns() - t0 > timeout_ns) {
          good = 0;
          break;
        }
      }
      good = __all_sync(0xffffffffu, good);
      if (good) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
          double sum = 0;
          for (int i = threadIdx.x; i < G; i += 32) sum += __ldcg(buf + (size_t)k * G + i);
          sum = warp_sum(sum);
          if (threadIdx.x == 0) res[k] = sum;
        }
      } else if (threadIdx.x == 0) {
        atomicExch(err, 1);
      }
      if (threadIdx.x == 0) ok = good;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = res[k];
    const bool r = ok != 0;
    __syncthreads();
    return r;
  }
};

// Writes this block's partial sums of NV values into buf (thread 0).
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* buf) {
  block_sum<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) buf[(size_t)k * gridDim.x + blockIdx.x] = v[k];
}

// Pipelined Jacobi-PCG (Ghysels & Vanroose 2014) with M = diag(Z)^-1:
//   g_i = (r_i,u_i), d_i = (w_i,u_i), m_i = M w_i, n_i = Z m_i
//   b_i = g_i/g_{i-1}, a_i = g_i/(d_i - b_i g_i/a_{i-1})   (b_0 = 0, a_0 = g_0/d_0)
//   z = n + b z,  q = m + b q,  s = w + b s,  p = u + b p
//   x += a p,  r -= a s,  u -= a q,  w -= a z
// Same iterates as standard PCG in exact arithmetic.  The dot products of
// iteration i are posted (partials + release-add on a counter) before the SpMV
// n_i = Z m_i and collected after it, so the reduction is off the critical
// path; blocks synchronise only with the blocks whose rows they gather
// (progress flags), never grid-wide.  A warp owns whole 32-row slices
// (lane = row) and streams them through shared memory (ChunkStream).
template <class VT>
__global__ void __launch_bounds__(kPcgThreads, 2) k_pcg(PcgArgs<VT> a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int n = a.n, nslices = (n + 31) >> 5;
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
  __syncthreads();

  BlockSync bs;
  bs.cnt = a.sync;
  bs.prog = a.sync + 1;
  bs.lo = a.nb_lo[blockIdx.x];
  bs.hi = a.nb_hi[blockIdx.x];
  bs.err = a.err;
  bs.timeout_ns = a.timeout_ns;

  VT* r = a.work;
  VT* u = r + n;
  VT* w = u + n;
  VT* z = w + n;
  VT* q = z + n;
  VT* s = q + n;
  VT* p = s + n;
  VT* nv = p + n;
  VT* mb[2] = {nv + n, nv + 2 * (size_t)n};
  const int G = gridDim.x;

  // P1: r = b - Z x0, u = M r (own rows)
  double bb = 0;
  for (int sl = st.s_begin; sl < st.s_end; sl++) {
    const int i = sl * 32 + lane;
    if (i >= n) continue;
    const double bi = (double)a.b[i];
    double ri = bi;
    if (a.warm) {
      const int b0 = __ldg(a.off + sl) + lane, wd = (__ldg(a.off + sl + 1) - __ldg(a.off + sl)) >> 5;
      VT acc = 0;
      for (int j = 0; j < wd; j++) acc += __ldg(a.val + b0 + 32 * j) * a.x[__ldg(a.col + b0 + 32 * j)];
      ri = bi - (double)acc;
    }
    const VT rv = (VT)ri;
    r[i] = rv;
    u[i] = rv * a.dinv[i];
    bb += bi * bi;
  }
  st.start(lane);
  bs.publish(1);
  if (!a.warm)
    for (int sl = st.s_begin; sl < st.s_end; sl++)
      if (sl * 32 + lane < n) a.x[sl * 32 + lane] = (VT)0;
  // P2: w = Z u, m0 = M w, dots of iteration 0
  bool alive = bs.wait_nb(1);
  if (!alive) st.failed = true;  // stop refilling: chunks may still be in flight
  double v[4] = {0, 0, 0, bb};
  for (int sl = st.s_begin; sl < st.s_end; sl++) {
    VT acc = 0;
    const int wd = (__ldg(a.off + sl + 1) - __ldg(a.off + sl)) >> 5;
    for (int c0 = 0; c0 < wd; c0 += kCh) {
      if (alive && st.wait(a.err, a.timeout_ns)) acc += chunk_dot<VT>(st.buf + st.nbc, min(kCh, wd - c0), lane, u);
      st.release(lane);
    }
    const int i = sl * 32 + lane;
    if (i < n) {
      w[i] = acc;
      mb[0][i] = acc * a.dinv[i];
      z[i] = (VT)0;
      q[i] = (VT)0;
      s[i] = (VT)0;
      p[i] = (VT)0;
      const double ri = (double)r[i], ui = (double)u[i];
      v[0] += ri * ui;
      v[1] += (double)acc * ui;
      v[2] += ri * ri;
    }
  }
  block_partials<4>(v, a.part);
  bs.publish(2);
  bs.arrive();

  double bnorm = 0, tol = 0, rn = 0, gam_old = 1, alpha_old = 1;
  int its = 0, status = 1;
  for (int i = 0;; i++) {
    // n_i = Z m_i  (neighbours' m_i published at phase i + 2)
    if (alive) alive = bs.wait_nb((unsigned)i + 2);
    if (!alive) st.failed = true;
    const VT* mi = mb[i & 1];
    for (int sl = st.s_begin; sl < st.s_end; sl++) {
      VT acc = 0;
      const int wd = (__ldg(a.off + sl + 1) - __ldg(a.off + sl)) >> 5;
      for (int c0 = 0; c0 < wd; c0 += kCh) {
        if (alive && st.wait(a.err, a.timeout_ns)) acc += chunk_dot<VT>(st.buf + st.nbc, min(kCh, wd - c0), lane, mi);
        st.release(lane);
      }
      const int ii = sl * 32 + lane;
      if (ii < n) nv[ii] = acc;
    }
    // reduction of iteration i (posted before the SpMV)
    double red[4];
    if (!alive || !bs.wait_red<4>((unsigned)(i + 1) * (unsigned)G, a.part + (size_t)(i & 1) * 4 * G, red)) {
      status = 3;
      break;
    }
    if (i == 0) {
      bnorm = sqrt(red[3]);
      tol = a.rtol * bnorm;
    }
    rn = sqrt(red[2]);
    if (!isfinite(bnorm) || !isfinite(rn)) { status = 2; break; }
    if (bnorm == 0.0) {
      for (int sl = st.s_begin; sl < st.s_end; sl++)
        if (sl * 32 + lane < n) a.x[sl * 32 + lane] = (VT)0;
      rn = 0;
      status = 0;
      break;
    }
    if (rn <= tol) { status = 0; break; }
    if (its >= a.maxit) { status = 1; break; }
    const double gam = red[0], del = red[1];
    const double beta = i > 0 ? gam / gam_old : 0.0;
    const double alpha = i > 0 ? gam / (del - beta * gam / alpha_old) : gam / del;
    gam_old = gam;
    alpha_old = alpha;
    const VT al = (VT)alpha, be = (VT)beta;
    VT* mnext = mb[(i + 1) & 1];
    double d[4] = {0, 0, 0, 0};
    for (int sl = st.s_begin; sl < st.s_end; sl++) {
      const int ii = sl * 32 + lane;
      if (ii >= n) continue;
      const VT zi = nv[ii] + be * z[ii];
      const VT qi = mi[ii] + be * q[ii];
      const VT si = w[ii] + be * s[ii];
      const VT pi = u[ii] + be * p[ii];
      const VT xi = a.x[ii] + al * pi;
      const VT ri = r[ii] - al * si;
      const VT ui = u[ii] - al * qi;
      const VT wi = w[ii] - al * zi;
      z[ii] = zi;
      q[ii] = qi;
      s[ii] = si;
      p[ii] = pi;
      a.x[ii] = xi;
      r[ii] = ri;
      u[ii] = ui;
      w[ii] = wi;
      mnext[ii] = wi * a.dinv[ii];
      d[0] += (double)ri * (double)ui;
      d[1] += (double)wi * (double)ui;
      d[2] += (double)ri * (double)ri;
    }
    its++;
    block_partials<4>(d, a.part + (size_t)((i + 1) & 1) * 4 * G);
    bs.publish((unsigned)i + 3);
    bs.arrive();
  }
  st.drain(a.timeout_ns);
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
    double q = 0;
    if (x) {  // x == null: x = 0, r = b without touching Z
      const int s = i >> 5, l = i & 31;
      const int bb = __ldg(off + s) + l, w = (__ldg(off + s + 1) - __ldg(off + s)) >> 5;
#pragma unroll 4
      for (int j = 0; j < w; j++) q += __ldcs(val + bb + 32 * j) * __ldg(x + __ldcs(col + bb + 32 * j));
    }
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
  const size_t smem = pcg_smem_bytes<VT>();
  cudaFuncSetAttribute(k_pcg<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<VT>, kPcgThreads, smem);
  long long cap = (long long)sms * (per_sm > 0 ? per_sm : 1);
  long long want = ((long long)n + kPcgThreads - 1) / kPcgThreads;  // one row per thread at most
  if (want < 1) want = 1;
  return (int)std::min(cap, want);
}

void pcg_neighbor_ranges(int n, int grid, const int* first, const int* last, int* lo, int* hi) {
  const int ns = (n + 31) / 32;
  const long long W = (long long)grid * kPcgWarps;
  std::vector<int> owner(ns);
  for (int b = 0; b < grid; b++) {
    const int s0 = (int)(ns * (kPcgWarps * (long long)b) / W), s1 = (int)(ns * (kPcgWarps * (long long)(b + 1)) / W);
    for (int s = s0; s < s1; s++) owner[s] = b;
  }
  for (int b = 0; b < grid; b++) {
    const int s0 = (int)(ns * (kPcgWarps * (long long)b) / W), s1 = (int)(ns * (kPcgWarps * (long long)(b + 1)) / W);
    int cmin = n, cmax = -1;
    for (int s = s0; s < s1; s++) {
      // the slice's stored columns: every row's own, and column 0 as the
      // padding of its empty rows (rows past n included) when any row of
      // the slice is non-empty
      int w = 0;
      bool empty_row = false;
      for (int r = 32 * s; r < 32 * s + 32; r++) {
        const bool has = r < n && last[r] >= first[r];
        w = std::max(w, has ? 1 : 0);
        empty_row = empty_row || !has;
        if (has) {
          cmin = std::min(cmin, first[r]);
          cmax = std::max(cmax, last[r]);
        }
      }
      if (w > 0 && empty_row) {
        cmin = std::min(cmin, 0);
        cmax = std::max(cmax, 0);
      }
    }
    if (cmax < 0) {
      lo[b] = b;
      hi[b] = b - 1;  // no neighbours
    } else {
      lo[b] = owner[cmin / 32];
      hi[b] = owner[cmax / 32];
    }
  }
}

template <class VT>
cudaError_t launch_pcg(const PcgArgs<VT>& a, int grid, cudaStream_t s) {
  PcgArgs<VT> args = a;
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel((const void*)k_pcg<VT>, dim3(grid), dim3(kPcgThreads), params,
                                     pcg_smem_bytes<VT>(), s);
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
