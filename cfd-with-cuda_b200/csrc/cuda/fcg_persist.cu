// Persistent two-level flexible CG: the iterations of an FP32 inner pressure
// solve on a structured grid (identity numbering, the 125-tap structured
// form of Z, the coarse space of coarse.cu) in one cooperative launch,
// instead of five dependent kernels per iteration replayed from a graph.
//
// One iteration, as the kernel sequence of fcg.cu / coarse.cu computes it:
//
//   c = P^T r                                   restriction      (1)
//   e = Zc^-1 c                                 coarse solve     (2)
//   z = D^-1 r + P e                            own rows         (3)
//   w = Z z, dots (z,w) (z,r) (z,q_j) (p_j,r)   structured SpMV  (4)
//   beta_j, alpha from the dots                 every block      (5)
//   p = z - sum beta_j p_j, q = w - sum beta_j q_j,
//   x += alpha p, r -= alpha q, (r,r)           own rows         (6)
//   convergence, iteration-limit and stall tests                 (7)
//
// Synchronisation (every wait bounded, a timeout raises *err and ends the
// solve with status 3): (1) needs all of r, (2) all of c, (3) all of e,
// (5) every block's dot partials, (7) every block's (r,r) partial: four
// grid-wide arrival points per iteration on one monotonic counter
// (release-add, acquire-poll).  (4) gathers z two grid planes either side,
// so a block waits only for the blocks owning those rows (progress flags).
// Every block sums the posted partials in the same fixed order (FP64) and
// takes the same decisions; partial buffers alternate between two halves,
// so a block can overwrite one only after every block has read it.
//
// Data written during the launch by other blocks (r, c, e, z) is read with
// plain loads after the acquiring wait; matrix data with read-only loads.
// The state words sc[] are read by every block at entry and written back by
// block 0 after the last arrival point.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "fcg_common.cuh"
#include "kernels.h"
#include "sell_stream.cuh"

namespace cfd {

namespace {

constexpr int kRestrictLines2 = 1024;  // y-z support lines of a coarse pair at most

// Arrives at grid-wide point `target / gridDim.x` and waits (thread 0,
// bounded) until every block has; false when the wait gave up or another
// block raised *err.  The caller's writes before the call are visible to
// every block after it.
__device__ __forceinline__ bool grid_point(unsigned* cnt, unsigned target, int* err, unsigned long long timeout_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    red_add_release_u32(cnt, 1u);
    int ok = 1;
    const unsigned long long t0 = global_ns();
    while (ld_acquire_u32(cnt) < target) {
      if (ld_volatile_i32(err) || global_ns() - t0 > timeout_ns) {
        ok = 0;
        break;
      }
    }
    if (!ok) atomicExch(err, 1);
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sum over all blocks of NV posted partials (buf[k * G + block]), the same
// fixed order in every block; valid in every thread.
template <int NV>
__device__ __forceinline__ void sum_posted(const double* buf, double (&v)[NV]) {
  __shared__ double res[NV];
  const int G = gridDim.x;
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double s = 0;
      for (int i = threadIdx.x; i < G; i += 32) s += __ldcg(buf + (size_t)k * G + i);
      s = warp_sum(s);
      if (threadIdx.x == 0) res[k] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = res[k];
  __syncthreads();
}

// Block partials of NV values into buf[k * G + block] (thread 0 writes).
template <int NV>
__device__ __forceinline__ void post_block(double (&v)[NV], double* buf) {
  block_sum<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) buf[(size_t)k * gridDim.x + blockIdx.x] = v[k];
}

// This block's own rows of phase k are written (progress flag).
__device__ __forceinline__ void publish(unsigned* prog, unsigned k) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release_u32(prog + blockIdx.x, k);
  }
}

// Waits (warp 0, bounded) until blocks lo..hi have published phase k.  The
// decision to stop polling is taken by the whole warp at once.
__device__ __forceinline__ bool wait_blocks(const unsigned* prog, int lo, int hi, unsigned k, int* err,
                                            unsigned long long timeout_ns) {
  __shared__ int s_ok;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    bool good = true;
    const unsigned long long t0 = global_ns();
    for (int j0 = lo; j0 <= hi && good; j0 += 32) {
      const int j = j0 + lane;
      bool done = j > hi;
      for (;;) {
        if (!done) done = ld_acquire_u32(prog + j) >= k;
        if (__all_sync(0xffffffffu, done)) break;
        if (__any_sync(0xffffffffu, ld_volatile_i32(err) != 0 || global_ns() - t0 > timeout_ns)) {
          good = false;
          break;
        }
      }
    }
    __threadfence();
    if (lane == 0) {
      if (!good) atomicExch(err, 1);
      s_ok = good;
    }
  }
  __syncthreads();
  return s_ok != 0;
}

// c = P^T r for one coarse (iy, iz) pair (the separable restriction of
// coarse.cu's k_restrict, with its scratch in the caller's shared memory).
__device__ void restrict_pair(const CoarseArgs<float>& a, const float* r, float* c, int pair,
                              unsigned char* scratch) {
  double* swt = reinterpret_cast<double*>(scratch);
  int* sbase = reinterpret_cast<int*>(swt + kRestrictLines2);
  double* sline = reinterpret_cast<double*>(sbase + kRestrictLines2);
  const int cx = a.cd[0], cy = a.cd[1];
  const int iy = pair % cy, iz = pair / cy;
  const int y0 = __ldg(a.ry + 2 * iy), ny = __ldg(a.ry + 2 * iy + 1) - y0 + 1;
  const int z0 = __ldg(a.rz + 2 * iz), nz = __ldg(a.rz + 2 * iz + 1) - z0 + 1;
  const int fx = a.fd[0], fxy = a.fd[0] * a.fd[1];
  const int nl = ny * nz;
  for (int l = threadIdx.x; l < nl; l += blockDim.x) {
    const int y = y0 + l % ny, z = z0 + l / ny;
    const int i0y = __ldg(a.i0y + y), i0z = __ldg(a.i0z + z);
    const double fy = __ldg(a.fy + y), fz = __ldg(a.fz + z);
    const double wy = i0y == iy ? 1.0 - fy : (i0y + 1 == iy ? fy : 0.0);
    const double wz = i0z == iz ? 1.0 - fz : (i0z + 1 == iz ? fz : 0.0);
    swt[l] = wy * wz;
    sbase[l] = fx * y + fxy * z;
  }
  __syncthreads();
  const int G = fx <= (int)blockDim.x ? (int)blockDim.x / fx : 1;
  const int g = threadIdx.x / fx;
  for (int x = threadIdx.x % fx; g < G && x < fx; x += (G == 1 ? (int)blockDim.x : fx)) {
    double acc = 0.0;
#pragma unroll 4
    for (int l = g; l < nl; l += G) acc += swt[l] * (double)r[sbase[l] + x];
    sline[g * fx + x] = acc;
    if (G != 1) break;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int ix = warp; ix < cx; ix += blockDim.x >> 5) {
    const int x0 = __ldg(a.rx + 2 * ix), x1 = __ldg(a.rx + 2 * ix + 1);
    double acc = 0.0;
    for (int x = x0 + lane; x <= x1; x += 32) {
      const int i0x = __ldg(a.i0x + x);
      const double fxw = __ldg(a.fx + x);
      const double wx = i0x == ix ? 1.0 - fxw : (i0x + 1 == ix ? fxw : 0.0);
      double sx = 0.0;
      for (int gg = 0; gg < G; gg++) sx += sline[gg * fx + x];
      acc += wx * sx;
    }
    acc = warp_sum(acc);
    if (lane == 0) c[ix + cx * (iy + cy * iz)] = (float)acc;
  }
  __syncthreads();
}

// 16-byte asynchronous copy global -> shared with an L2 cache policy
__device__ __forceinline__ void cp_async16_hint(void* dst, const void* src, unsigned long long policy) {
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "l"(policy)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// sum of 8 FP16 entries packed in q times 8 FP32 values in shared memory
__device__ __forceinline__ float dot8_smem(const uint4& q, const float* c) {
  const __half2* h = reinterpret_cast<const __half2*>(&q);
  const float4 c0 = reinterpret_cast<const float4*>(c)[0], c1 = reinterpret_cast<const float4*>(c)[1];
  const float2 f0 = __half22float2(h[0]), f1 = __half22float2(h[1]), f2 = __half22float2(h[2]),
               f3 = __half22float2(h[3]);
  return (f0.x * c0.x + f0.y * c0.y) + (f1.x * c0.z + f1.y * c0.w) + (f2.x * c1.x + f2.y * c1.y) +
         (f3.x * c1.z + f3.y * c1.w);
}

constexpr int kStChunkBytes = kStTaps * 32 * (int)sizeof(float);

template <int MD>
__global__ void __launch_bounds__(kPcgThreads, 2) k_fcg2l(FcgArgs<float> a, CoarseArgs<float> ca, Fcg2lArgs pa) {
  if (ld_volatile_i32(a.st.done)) return;
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int NV = fcg_parts<MD>();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int G = gridDim.x;
  const int n = a.n, fx = a.fd[0], fy = a.fd[1], fxy = a.fd[0] * a.fd[1];
  const int nslices = (n + 31) >> 5;
  const int W = G * kPcgWarps, gw = blockIdx.x * kPcgWarps + wib;
  const int s0 = (int)((long long)nslices * gw / W), s1 = (int)((long long)nslices * (gw + 1) / W);
  float* buf = reinterpret_cast<float*>(smem) + (size_t)wib * kStBuf * kStTaps * 32;
  unsigned long long* mbar =
      reinterpret_cast<unsigned long long*>(smem + (size_t)kPcgWarps * kStBuf * kStChunkBytes) + wib * kStBuf;
  if (lane == 0)
    for (int b = 0; b < kStBuf; b++) mbar_init(mbar + b, 1);
  mbar_init_fence();
  __syncthreads();

  // solve state, identical in every block, in shared memory: thread 0
  // forms the coefficients and runs the tests, the block reads them back
  __shared__ double st[kFcgScalars];
  __shared__ int s_status;
  if (threadIdx.x < kFcgScalars) st[threadIdx.x] = a.st.sc[threadIdx.x];
  if (threadIdx.x == 0) s_status = -1;
  __syncthreads();
  const int m = (int)st[kFcgM], anchor = (int)st[kFcgAnchor];
  int it = (int)st[kFcgIt];
  const int lo = __ldg(pa.nb_lo + blockIdx.x), hi = __ldg(pa.nb_hi + blockIdx.x);
  unsigned* cnt = pa.sync;
  unsigned* prog = pa.sync + 1;
  int* err = a.st.err;
  const unsigned long long tmo = a.st.timeout_ns;
  const int reach = 2 + 2 * fx + 2 * fxy;
  const size_t nn = (size_t)n;
  float* r = a.r;
  float* z = a.z;
  float* w = a.w;
  unsigned point = 0;  // grid-wide arrival points passed
  int kbase = 0;       // this warp's matrix chunks issued in earlier passes
  int pend_lo = 0, pend_hi = 0;  // chunks issued but not yet consumed [pend_lo, pend_hi)
  // phase times of block 0 (thread 0) into pa.timing
  __shared__ unsigned long long s_tc;
  if (threadIdx.x == 0) s_tc = global_ns();
  auto lap = [&](int k) {
    if (pa.timing && blockIdx.x == 0 && threadIdx.x == 0) {
      const unsigned long long t = global_ns();
      pa.timing[k] += (double)(t - s_tc);
      s_tc = t;
    }
  };

  for (;;) {
    // (1) c = P^T r
    for (int pair = blockIdx.x; pair < ca.cd[1] * ca.cd[2]; pair += G) restrict_pair(ca, r, pa.c, pair, smem);
    lap(0);
    if (!grid_point(cnt, ++point * (unsigned)G, err, tmo)) break;
    // (2) e = Zc^-1 c: c staged in shared memory; each row of the FP16
    // inverse split into pa.pieces pieces, a warp per piece: the piece is
    // copied into the warp's shared-memory buffer by 16-byte asynchronous
    // copies (about ten in flight per lane) and multiplied with c there.
    // Piece p of row r goes to pa.e[p * nc + r]; (3) sums the pieces in
    // order, so the result does not depend on which warp finishes first.
    {
      const unsigned long long keep = l2_evict_last();
      const float rscale = (float)(1.0 / ca.inv_scale);
      float* cs = reinterpret_cast<float*>(smem);
      for (int k = threadIdx.x; k < ca.nc; k += blockDim.x) cs[k] = __ldcg(pa.c + k);
      for (int k = ca.nc + threadIdx.x; k < ca.ldinv; k += blockDim.x) cs[k] = 0.f;
      __syncthreads();
      const int nv8 = ca.ldinv >> 3, P = pa.pieces;
      const int plen = (nv8 + P - 1) / P;  // 16-byte groups per piece
      uint4* pb = reinterpret_cast<uint4*>(smem + ((ca.ldinv * 4 + 15) & ~15)) + (size_t)wib * plen;
      for (int item = gw; item < P * ca.nc; item += W) {
        const int row = item / P, piece = item % P;
        const int j0 = piece * plen, j1 = min(nv8, j0 + plen);
        const uint4* ir = reinterpret_cast<const uint4*>(ca.inv16 + (size_t)row * ca.ldinv);
        for (int j = j0 + lane; j < j1; j += 32) cp_async16_hint(pb + (j - j0), ir + j, keep);
        cp_async_wait_all();  // this lane's own copies; it reads only those
        float acc = 0.f;
        for (int j = j0 + lane; j < j1; j += 32) acc += dot8_smem(pb[j - j0], cs + 8 * j);
        acc = warp_sum(acc);
        if (lane == 0) pa.e[(size_t)piece * ca.nc + row] = acc * rscale;
        __syncwarp();
      }
    }
    // the first chunks of this iteration's matrix stream go out now and
    // arrive during (3) and the neighbour wait (the scratch of (1)-(2) and
    // the chunk buffers share shared memory)
    __syncthreads();
    const int total = (s1 - s0) * 5;  // chunks of this warp per pass
    auto issue = [&](int k) {         // chunk k of this pass
      if (lane == 0 && k < total) {
        const unsigned long long once = l2_evict_first();
        const int b = (kbase + k) % kStBuf;
        const float* src = a.stencil + ((size_t)(s0 + k / 5) * 125 + (k % 5) * kStTaps) * 32;
        fence_proxy_async_smem();
        mbar_expect_tx(mbar + b, kStChunkBytes);
        bulk_g2s_hint(buf + (size_t)b * kStTaps * 32, src, kStChunkBytes, mbar + b, once);
      }
    };
    for (int k = 0; k < kStBuf; k++) issue(k);
    pend_lo = kbase;
    pend_hi = kbase + min(kStBuf, total);
    lap(1);
    if (!grid_point(cnt, ++point * (unsigned)G, err, tmo)) break;
    // (3) z = D^-1 r + P e on this warp's rows
    {
    const int cx = ca.cd[0], cxy = ca.cd[0] * ca.cd[1];
    const int bx = ca.cd[0] > 1, by = ca.cd[1] > 1, bz = ca.cd[2] > 1;
#pragma unroll 4
    for (int sl = s0; sl < s1; sl++) {
      const int i = sl * 32 + lane;
      if (i >= n) continue;
      const int x = i % fx, y = (i / fx) % fy, zz = i / fxy;
      const int ix = __ldg(ca.i0x + x), iy = __ldg(ca.i0y + y), iz = __ldg(ca.i0z + zz);
      const float wx = (float)__ldg(ca.fx + x), wy = (float)__ldg(ca.fy + y), wz = (float)__ldg(ca.fz + zz);
      const float* e0 = pa.e + ix + cx * iy + cxy * iz;
      float pe = 0.f;
#pragma unroll
      for (int cnr = 0; cnr < 8; cnr++) {
        const int dx = cnr & 1, dy = (cnr >> 1) & 1, dz = cnr >> 2;
        if ((dx && !bx) || (dy && !by) || (dz && !bz)) continue;
        const float wt = (dx ? wx : 1 - wx) * (dy ? wy : 1 - wy) * (dz ? wz : 1 - wz);
        const float* ep = e0 + dx + cx * dy + cxy * dz;
        float ev = ep[0];
        for (int q = 1; q < pa.pieces; q++) ev += ep[(size_t)q * ca.nc];
        pe += wt * ev;
      }
      z[i] = __ldg(a.dinv + i) * r[i] + pe;
    }
    }
    lap(2);
    publish(prog, (unsigned)it + 1);
    if (!wait_blocks(prog, lo, hi, (unsigned)it + 1, err, tmo)) break;
    lap(3);
    const unsigned long long t_spmv = threadIdx.x == 0 ? global_ns() : 0;
    // (4) w = Z z with the dot products; chunk k of the pass is the warp's
    // chunk kbase + k since launch, in buffer (kbase + k) % kStBuf, whose
    // completion is that buffer's phase (kbase + k) / kStBuf
    const int nd = it < m ? it : m;
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = 0.0;
    bool ok = true;
    {
      int k = 0;
      for (int sl = s0; sl < s1 && ok; sl++) {
        const int i = sl * 32 + lane;
        const bool inside = sl * 32 >= reach && sl * 32 + 31 + reach < n;
        float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        for (int dz = -2; dz <= 2 && ok; dz++, k++) {
          const int K = kbase + k, b = K % kStBuf;
          if (!__all_sync(0xffffffffu, mbar_wait_bounded(mbar + b, (unsigned)((K / kStBuf) & 1), tmo))) {
            ok = false;
            if (lane == 0) atomicExch(err, 1);
            break;
          }
          const float* q = buf + (size_t)b * kStTaps * 32 + lane;
          if (inside)
            stencil_plane_shfl<false, false>(q, z, i + fxy * dz, fx, n, lane, acc);
          else
            stencil_plane_shfl<true, false>(q, z, i + fxy * dz, fx, n, lane, acc);
          __syncwarp();
          pend_lo = K + 1;
          issue(k + kStBuf);
          if (k + kStBuf < total) pend_hi = kbase + k + kStBuf + 1;
        }
        if (ok && i < n) fcg_row_dots<MD>(a, i, z[i], ((acc[0] + acc[1]) + (acc[2] + acc[3])) + acc[4], nd, v);
      }
    }
    kbase += total;
    // a chunk wait gave up in some warp: the whole block leaves together,
    // and the other blocks learn it from *err at their next wait
    if (!__syncthreads_and(ok)) break;
    if (pa.tblock && threadIdx.x == 0) pa.tblock[blockIdx.x] += (double)(global_ns() - t_spmv);
    lap(4);
    ++point;
    post_block<NV>(v, pa.part + (size_t)(point & 1) * NV * G);
    if (!grid_point(cnt, point * (unsigned)G, err, tmo)) break;
    sum_posted<NV>(pa.part + (size_t)(point & 1) * NV * G, v);
    lap(5);
    // (5) coefficients (thread 0; the same values in every block)
    const int slot = fcg_slot(it, m, anchor);
    if (threadIdx.x == 0) {
      double pq = v[0], pr = v[1];
      bool bad = false;
#pragma unroll
      for (int j = 0; j < MD; j++) {
        double bj = 0.0;
        if (j < nd) {
          bj = v[2 + j] / st[kFcgPQ0 + j];
          pq -= bj * v[2 + j];
          pr -= bj * v[2 + MD + j];
          bad = bad || !isfinite(bj);
        }
        st[kFcgBeta0 + j] = bj;
      }
      const double alpha = pr / pq;
      bad = bad || !(pq > 0.0) || !isfinite(alpha);
      st[kFcgAlpha] = alpha;
      if (bad)
        s_status = isfinite(v[0]) ? 4 : 2;  // breakdown
      else
        st[kFcgPQ0 + slot] = pq;
    }
    __syncthreads();
    if (s_status >= 0) break;
    // (6) update of this warp's rows
    {
      const float al = (float)st[kFcgAlpha];
      float be[MD];
#pragma unroll
      for (int j = 0; j < MD; j++) be[j] = (float)st[kFcgBeta0 + j];
      double d[1] = {0.0};
#pragma unroll 4
      for (int sl = s0; sl < s1; sl++) {
        const int i = sl * 32 + lane;
        if (i >= n) continue;
        float pi = z[i], qi = w[i];
#pragma unroll
        for (int j = 0; j < MD; j++) {
          if (j < nd) {
            pi -= be[j] * a.p[j * nn + i];
            qi -= be[j] * a.q[j * nn + i];
          }
        }
        a.p[slot * nn + i] = pi;
        a.q[slot * nn + i] = qi;
        a.x[i] += al * pi;
        const float ri = r[i] - al * qi;
        r[i] = ri;
        d[0] += (double)ri * ri;
      }
      ++point;
      post_block<1>(d, pa.part + (size_t)(point & 1) * NV * G);
      if (!grid_point(cnt, point * (unsigned)G, err, tmo)) break;
      sum_posted<1>(pa.part + (size_t)(point & 1) * NV * G, d);
      if (threadIdx.x == 0) st[kFcgRR] = d[0];
    }
    lap(6);
    // (7) tests, as k_fcg_update
    it = it + 1;
    if (threadIdx.x == 0) {
      const double rr = st[kFcgRR], itn = it, window = st[kFcgWindow];
      const bool mark = window > 0 && fmod(itn, window) == 0.0;
      int status = -1;
      if (!isfinite(rr))
        status = 2;
      else if (rr <= st[kFcgRtol] * st[kFcgRtol] * st[kFcgBB])
        status = 0;
      else if (itn >= st[kFcgMaxit])
        status = 1;
      else if (mark && rr > st[kFcgStall2] * st[kFcgRRMark])
        status = 4;
      if (status < 0 && mark) st[kFcgRRMark] = rr;
      s_status = status;
    }
    __syncthreads();
    if (s_status >= 0) break;
  }
  // copies still in flight into this block's shared memory (only after a
  // wait gave up): one more bounded wait each before the block ends
  if (lane == 0)
    for (int K = pend_lo; K < pend_hi; K++) mbar_wait_bounded(mbar + K % kStBuf, (unsigned)((K / kStBuf) & 1), tmo);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // the loop ended on a test (s_status >= 0) or on a wait that gave up
    const int status = (s_status < 0 || ld_volatile_i32(err)) ? 3 : s_status;
    double* sc = a.st.sc;
    st[kFcgIt] = it;
    st[kFcgStatus] = status;
    for (int k = 0; k < kFcgScalars; k++) sc[k] = st[k];
    a.st.done[0] = 1;
  }
}

}  // namespace

size_t fcg2l_smem_bytes() { return stencil_smem_bytes<float>(); }

int fcg2l_grid(int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int smem = (int)fcg2l_smem_bytes();
  cudaFuncSetAttribute(k_fcg2l<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(k_fcg2l<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(k_fcg2l<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int occ[3] = {0, 0, 0};
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_fcg2l<1>, kPcgThreads, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_fcg2l<2>, kPcgThreads, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], k_fcg2l<4>, kPcgThreads, smem);
  per_sm = std::min(std::min(occ[0], occ[1]), std::min(occ[2], 2));
  return sms * per_sm;
}

void fcg2l_neighbor_ranges(int n, int grid, int reach, int* lo, int* hi) {
  const int ns = (n + 31) / 32;
  const long long W = (long long)grid * kPcgWarps;
  auto first_slice = [&](int b) { return (int)((long long)ns * (kPcgWarps * (long long)b) / W); };
  std::vector<int> owner(ns);
  for (int b = 0; b < grid; b++)
    for (int s = first_slice(b); s < first_slice(b + 1); s++) owner[s] = b;
  for (int b = 0; b < grid; b++) {
    const int r0 = first_slice(b) * 32, r1 = std::min(n, first_slice(b + 1) * 32);
    if (r0 >= r1) {
      lo[b] = b;
      hi[b] = b - 1;
      continue;
    }
    lo[b] = owner[std::max(0, r0 - reach) / 32];
    hi[b] = owner[std::min(n - 1, r1 - 1 + reach) / 32];
  }
}

int fcg2l_pieces(int ldinv) {
  const size_t cbytes = ((size_t)ldinv * 4 + 15) & ~(size_t)15, nv8 = (size_t)ldinv / 8;
  for (int p = 1; p <= 4; p *= 2)
    if (cbytes + (size_t)kPcgWarps * ((nv8 + p - 1) / p) * 16 <= (size_t)kPcgWarps * kStBuf * kStChunkBytes) return p;
  return 0;
}

cudaError_t launch_fcg2l(const FcgArgs<float>& a, const CoarseArgs<float>& ca, const Fcg2lArgs& pa, int grid,
                         cudaStream_t s) {
  if (pa.pieces < 1 || pa.pieces != fcg2l_pieces(ca.ldinv)) return cudaErrorInvalidValue;
  if (!a.stencil || ca.pmap || a.st.m < 1 || a.st.m > 4 || grid < 1) return cudaErrorInvalidValue;
  if ((long long)ca.fd[0] * ca.fd[1] * ca.fd[2] != a.n) return cudaErrorInvalidValue;
  if (ca.ldinv % 8 || ca.ldinv < ca.nc || (size_t)ca.ldinv * sizeof(float) > fcg2l_smem_bytes())
    return cudaErrorInvalidValue;
  if (ca.fd[0] > kPcgThreads) return cudaErrorInvalidValue;  // restriction scratch: one x-line per group
  for (int ax = 1; ax < 3; ax++) {
    const double h = ca.cd[ax] > 1 ? (double)(ca.fd[ax] - 1) / (ca.cd[ax] - 1) : 1.0;
    if ((2 * h + 1) * (2 * h + 1) > kRestrictLines2) return cudaErrorInvalidValue;
  }
  FcgArgs<float> aa = a;
  CoarseArgs<float> cc = ca;
  Fcg2lArgs pp = pa;
  void* params[] = {&aa, &cc, &pp};
  const void* fn = a.st.m == 1 ? (const void*)k_fcg2l<1> : (a.st.m == 2 ? (const void*)k_fcg2l<2> : (const void*)k_fcg2l<4>);
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kPcgThreads), params, fcg2l_smem_bytes(), s);
}

}  // namespace cfd
