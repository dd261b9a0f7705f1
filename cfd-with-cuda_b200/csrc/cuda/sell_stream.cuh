// Shared-memory staged streaming of a SELL-32 matrix (used by the
// persistent PCG kernel and the flexible-CG SpMV): each warp walks its own
// contiguous range of 32-row slices as a cyclic stream of chunks (kCh
// columns x 32 rows of column indices and values).  Lane 0 keeps kNbuf<VT>
// chunks in flight with bulk asynchronous copies completed on one mbarrier
// per buffer, so address generation never stalls the loads.  Every wait is
// bounded.
#pragma once
#include "common.cuh"

namespace cfd {
namespace {

constexpr int kPcgWarps = 16;
constexpr int kPcgThreads = kPcgWarps * 32;

// The stream repeats cyclically, so in the persistent PCG the copies for the
// next iteration's first chunks are already in flight while the warp waits
// at the grid barrier; a single pass drains the wrapped copies at its end.
constexpr int kCh = 8;
// chunk buffers per warp: three FP32 or two FP64 chunks keep two blocks of
// 16 warps per SM within the shared-memory budget
template <class VT>
constexpr int kNbuf = sizeof(VT) == 4 ? 3 : 2;

template <class VT>
struct __align__(16) Chunk {
  int col[kCh * 32];
  VT val[kCh * 32];
};

template <class VT>
constexpr size_t pcg_smem_bytes() {
  return (size_t)kPcgWarps * kNbuf<VT> * (sizeof(Chunk<VT>) + sizeof(unsigned long long));
}

template <class VT>
struct ChunkStream {
  const int* off;
  const int* col;
  const VT* val;
  Chunk<VT>* buf;               // kNbuf<VT> buffers of this warp
  unsigned long long* mbar;     // kNbuf<VT> mbarriers of this warp
  int s_begin, s_end;           // owned slices [s_begin, s_end)
  int is, ik, nbi;              // next chunk to issue (slice, chunk, buffer)
  int cs, ck, nbc;              // next chunk to consume
  unsigned parity;              // phase parity per buffer (bit b)
  bool failed;

  __device__ int nchunks(int s) const { return ((__ldg(off + s + 1) - __ldg(off + s)) / 32 + kCh - 1) / kCh; }

  __device__ void issue(int lane) {
    if (lane == 0) {
      const int base = __ldg(off + is), w = (__ldg(off + is + 1) - base) >> 5;
      const int c0 = ik * kCh, nc = min(kCh, w - c0);
      Chunk<VT>* B = buf + nbi;
      fence_proxy_async_smem();
      mbar_expect_tx(mbar + nbi, (unsigned)(nc * 32 * (4 + (int)sizeof(VT))));
      bulk_g2s(B->col, col + base + c0 * 32, (unsigned)(nc * 32 * 4), mbar + nbi);
      bulk_g2s(B->val, val + base + c0 * 32, (unsigned)(nc * 32 * (int)sizeof(VT)), mbar + nbi);
    }
    if (++ik == nchunks(is)) {
      ik = 0;
      if (++is == s_end) is = s_begin;
    }
    nbi = (nbi + 1 == kNbuf<VT>) ? 0 : nbi + 1;
  }

  __device__ void start(int lane) {
    if (s_begin < s_end)
      for (int k = 0; k < kNbuf<VT>; k++) issue(lane);
  }

  // Waits for the next chunk; false (and *err set) when the bounded wait gave up.
  __device__ bool wait(int* err, unsigned long long timeout_ns) {
    if (failed) return false;
    if (!mbar_wait_bounded(mbar + nbc, (parity >> nbc) & 1u, timeout_ns)) {
      failed = true;
      atomicExch(err, 1);
      return false;
    }
    return true;
  }

  // Releases the consumed buffer, refills it, advances; true at slice end.
  __device__ bool release(int lane) {
    __syncwarp();
    parity ^= 1u << nbc;
    nbc = (nbc + 1 == kNbuf<VT>) ? 0 : nbc + 1;
    if (!failed) issue(lane);
    if (++ck == nchunks(cs)) {
      ck = 0;
      if (++cs == s_end) cs = s_begin;
      return true;
    }
    return false;
  }

  // Waits (bounded) for every copy still in flight before the block exits.
  __device__ void drain(unsigned long long timeout_ns) {
    if (s_begin >= s_end) return;
    for (int k = 0; k < kNbuf<VT>; k++) {
      const int b = (nbc + k) % kNbuf<VT>;
      if (!mbar_wait_bounded(mbar + b, (parity >> b) & 1u, timeout_ns)) break;
      parity ^= 1u << b;
    }
  }
};

// Product of one staged chunk with a gathered vector g.  Gathers are plain
// (L1-cached) loads: g is written by other blocks during the solve, and the
// release/acquire progress flags make those writes visible before use.
template <class VT>
__device__ __forceinline__ VT chunk_dot(const Chunk<VT>* B, int nc, int lane, const VT* g) {
  VT acc = 0;
#pragma unroll
  for (int jj = 0; jj < kCh; jj++)
    if (jj < nc) acc += B->val[jj * 32 + lane] * g[B->col[jj * 32 + lane]];
  return acc;
}

}  // namespace
}  // namespace cfd
