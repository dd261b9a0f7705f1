// Row-level pieces shared by the flexible-CG kernels (fcg.cu) and the
// persistent two-level solve (fcg_persist.cu): the per-row dot products of
// an iteration and the 125-tap structured SpMV of the pressure matrix.
#pragma once
#include "common.cuh"
#include "kernels.h"
#include "sell_stream.cuh"

namespace cfd {
namespace {

constexpr int kFcgThreads = 256;
// partial sums per block of an SpMV kernel instantiated for at most MD
// stored directions: (z,w), (z,r), (z,q_j), (p_j,r)
template <int MD>
__host__ __device__ constexpr int fcg_parts() {
  return 2 + 2 * MD;
}
constexpr int kFcgParts = fcg_parts<kFcgMaxM>();

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

// Per-row part of the SpMV kernels: w[i] and the dot products of the
// iteration (z,w) (z,r) (z,q_j) (p_j,r), accumulated into v.
template <int MD, class VT>
__device__ __forceinline__ void fcg_row_dots(const FcgArgs<VT>& a, int i, VT zv, VT wi, int nd,
                                             double (&v)[fcg_parts<MD>()]) {
  const size_t n = (size_t)a.n;
  a.w[i] = wi;
  const double zi = zv, ri = a.r[i];
  v[0] += zi * (double)wi;
  v[1] += zi * ri;
#pragma unroll
  for (int j = 0; j < MD; j++) {
    if (j < nd) {
      v[2 + j] += zi * (double)a.q[j * n + i];
      v[2 + MD + j] += (double)a.p[j * n + i] * ri;
    }
  }
}

// w = Z z on a structured grid of pressure nodes (identity numbering, node
// x + fx (y + fy z)): Z couples nodes within two grid steps per axis, so a
// row is 125 coefficients.  They are stored per 32-row slice, tap-major
// inside the slice (coef[slice][tap][lane], zero for couplings that do not
// exist): no column indices are streamed, and the gathers of z are
// contiguous across the warp.  Each warp owns a contiguous range of slices
// and streams it through shared memory in chunks of 25 taps (one dz plane,
// 3.2 KB), two chunks in flight per warp on bulk asynchronous copies.  Taps
// that leave the grid have zero coefficients.  Slices whose every tap stays
// inside [0, n) read z at i + dx + fx dy + fxy dz directly (five row
// pointers per plane, dx folded into the load offsets); the few slices
// within two planes of either end clamp the index.
constexpr int kStTaps = 25;
constexpr int kStBuf = 2;
template <class VT>
constexpr size_t stencil_smem_bytes() {
  return (size_t)kPcgWarps * kStBuf * (kStTaps * 32 * sizeof(VT) + sizeof(unsigned long long));
}

// One dz plane of a row (25 taps, coefficients q[t * 32] in shared memory)
// into the five per-dy accumulators.
template <bool CLAMP, class VT>
__device__ __forceinline__ void stencil_plane(const VT* q, const VT* __restrict__ z, int base, int fx, int n,
                                              VT (&acc)[5]) {
#pragma unroll
  for (int dy = -2; dy <= 2; dy++) {
    const int rb = base + fx * dy;
#pragma unroll
    for (int dx = -2; dx <= 2; dx++) {
      VT zv;
      if constexpr (CLAMP) {
        int j = rb + dx;
        j = j < 0 ? 0 : (j >= n ? n - 1 : j);
        zv = __ldg(z + j);
      } else {
        zv = __ldg(z + rb + dx);
      }
      acc[dy + 2] += q[((dy + 2) * 5 + dx + 2) * 32] * zv;
    }
  }
}

// The same plane with the gathers shared across the warp: the 32 rows of a
// slice are consecutive grid nodes, so lane l + dx holds z[rb(l) + dx] of
// lane l.  Lane l loads z[rb(l) - 2] and lanes 0..3 the four values past the
// warp's window; the five dx taps then come from shuffles.  Two loads per
// dy row instead of five, identical products and sums.  NC: read-only
// (non-coherent) loads, for a z that no thread of the launch writes.
template <bool NC, class VT>
__device__ __forceinline__ VT ld_z(const VT* z, int j) {
  if constexpr (NC) return __ldg(z + j);
  return z[j];
}
template <bool CLAMP, bool NC, class VT>
__device__ __forceinline__ void stencil_plane_shfl(const VT* q, const VT* __restrict__ z, int base, int fx, int n,
                                                   int lane, VT (&acc)[5]) {
#pragma unroll
  for (int dy = -2; dy <= 2; dy++) {
    const int rb = base + fx * dy;
    int j0 = rb - 2, j1 = rb + 30;
    if constexpr (CLAMP) {
      j0 = j0 < 0 ? 0 : (j0 >= n ? n - 1 : j0);
      j1 = j1 < 0 ? 0 : (j1 >= n ? n - 1 : j1);
    }
    const VT w0 = ld_z<NC>(z, j0);
    const VT w1 = lane < 4 ? ld_z<NC>(z, j1) : (VT)0;
#pragma unroll
    for (int dx = -2; dx <= 2; dx++) {
      VT zv;
      if (dx == -2) {
        zv = w0;
      } else {
        const int t = lane + dx + 2;
        const VT lo = __shfl_sync(0xffffffffu, w0, t & 31);
        const VT hi = __shfl_sync(0xffffffffu, w1, t & 31);
        zv = t < 32 ? lo : hi;
      }
      acc[dy + 2] += q[((dy + 2) * 5 + dx + 2) * 32] * zv;
    }
  }
}

}  // namespace
}  // namespace cfd
