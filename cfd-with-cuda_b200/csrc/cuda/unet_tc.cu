// Tensor-core (tcgen05) 3x3x3 convolution, stride 1 or 2, for the U-Net's
// inference path.
//
// Implicit GEMM without an im2col buffer.  A CTA owns a brick of output
// voxels; one thread brings the brick plus a one-voxel halo into shared
// memory with TMA tensor copies (zero-filled outside the grid), one plane
// per 8 input channels, each halo voxel one 16-byte row of the plane (rows
// numbered hx + HX (hy + HY hz) over the halo box, the order in which the
// tensor copy lays out its box).  In that numbering
// every tap (dx, dy, dz) is a constant row shift, so the A operand of tap k
// for 128 consecutive rows is the plane itself at a shifted start address:
// no data is copied per tap.  Rows that fall on the halo ring compute
// garbage that is never stored.  The weights of all 27 taps for the CTA's
// slice of output channels are resident in shared memory, pre-packed in the
// tensor core's canonical K-major layout and brought in by one bulk copy.
//
// Stride 2 (the U-Net's down-sampling layers) runs on the same machinery:
// the copies split the fine input into its 8 parity phases (voxel (2i+px,
// 2j+py, 2k+pz) -> phase px + 2py + 4pz at (i, j, k); a traversal stride of
// 2 along x, y and z), and tap d of output X
// reads phase (d != 0) at coarse index X + (d == -1 ? -1 : 0), again a
// constant row shift inside that phase's planes (low-side halo only).
//
// Lane 0 of every warp issues tcgen05.mma (M = 128 rows, N = output
// channels of the slice, K = 16 input channels) for its share of the CTA's
// tiles -- or, when a group has fewer tiles than warps, for its share of a
// tile's taps into its own TMEM accumulator (split K) -- and commits to its
// own mbarrier, so the per-instruction issue cost is spread over four
// issuers.  The warps read the accumulators back with tcgen05.ld (warp w
// owns rows 32w..32w+31), sum the split-K partials, add the bias, apply the
// activation and store BF16 (or FP32) channels-last.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "tcgen05.cuh"
#include "unet.h"

namespace cfd {

namespace {

constexpr int kTcThreads = 128;
constexpr int kTmemCols = 128;
constexpr unsigned long long kTcWaitNs = 2000000000ULL;

struct Dims6 {
  int c[3], f[3];
};

// BF16 x BF16 -> FP32, both operands K-major, M = 128.
__host__ __device__ constexpr unsigned umma_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                     unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// tcgen05.ld without its wait, for several loads in flight; tmem_wait_ld
// then waits for all of them, and reg_pin16 (an empty statement that
// "modifies" the registers, placed after the wait) keeps every use of the
// loaded registers after the wait.
__device__ __forceinline__ void tmem_ld16_async(unsigned taddr, unsigned (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void reg_pin16(unsigned (&r)[16]) {
  asm volatile(""
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]));
}

// One TMA tensor copy of a 4-D box (coordinates innermost first) into shared
// memory, completing on the mbarrier (no multicast).
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// The halo brick by TMA: one copy per (phase, 8-channel chunk), each a box
// of HX x HY x HZ voxels starting one voxel below the brick (stride 1), or
// at phase (px, py, pz) of the voxel pairs below it (stride 2: coordinate
// 2 (x0 - 1) + px with traversal stride 2).  Called by one thread after the
// expect_tx of their bytes on bar.
template <int NCH, int STRIDE>
__device__ __forceinline__ void load_halo(const ConvTcParams& p, unsigned char* A, int x0, int y0, int z0,
                                          unsigned long long* bar) {
  constexpr int NPH = STRIDE == 2 ? 8 : 1;
#pragma unroll 1
  for (int ph = 0; ph < NPH; ph++) {
    const int px = ph & 1, py = (ph >> 1) & 1, pz = ph >> 2;
    const int cx = STRIDE == 2 ? 2 * (x0 - 1) + px : x0 - 1;
    const int cy = STRIDE == 2 ? 2 * (y0 - 1) + py : y0 - 1;
    const int cz = STRIDE == 2 ? 2 * (z0 - 1) + pz : z0 - 1;
#pragma unroll
    for (int c = 0; c < NCH; c++)
      tma_load_4d(A + (size_t)(ph * NCH + c) * p.plane_bytes, &p.tmap, 8 * c, cx, cy, cz, bar);
  }
}

template <int CIN, int STRIDE>
__global__ void __launch_bounds__(kTcThreads) k_conv_tc(const __grid_constant__ ConvTcParams p) {
  constexpr int NCH = CIN / 8, KSTEPS = CIN / 16, NPH = STRIDE == 2 ? 8 : 1;
  constexpr int NWARP = kTcThreads / 32;
  if (p.skip && *p.skip) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* A = smem;
  unsigned char* W = smem + (size_t)NPH * NCH * p.plane_bytes;
  const unsigned wbytes = 27u * CIN * p.N * 2u;
  // barrier 0: weights; barrier 1 + w: MMAs issued by warp w
  unsigned long long* bars = (unsigned long long*)(W + wbytes);  // wbytes is a multiple of 16
  unsigned* tmem_slot = (unsigned*)(bars + 1 + NWARP);
  float* sbias = (float*)(tmem_slot + 2);  // N floats

  const int b = blockIdx.x, slice = blockIdx.y;
  const int bx = b % p.nb[0], by = (b / p.nb[0]) % p.nb[1], bz = b / (p.nb[0] * p.nb[1]);
  const int x0 = bx * p.brick[0], y0 = by * p.brick[1], z0 = bz * p.brick[2];
  const int HX = p.halo[0], HY = p.halo[1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i <= NWARP; i++) mbar_init(&bars[i], 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  for (int i = threadIdx.x; i < p.N; i += blockDim.x) {
    const int co = slice * p.N + i;
    sbias[i] = co < p.cout ? p.bias[co] : 0.f;
  }
  if (threadIdx.x == 0) {
    const unsigned abytes = (unsigned)NPH * NCH * 16u * (unsigned)(HX * HY * p.halo[2]);
    mbar_expect_tx(&bars[0], wbytes + abytes);
    bulk_g2s(W, p.wpack + (size_t)slice * 27 * CIN * p.N, wbytes, &bars[0]);
    load_halo<NCH, STRIDE>(p, A, x0, y0, z0, &bars[0]);
  }
  {
    // rows past the halo box that tap shifts of the last tiles can read: zeros
    const int nbox = HX * HY * p.halo[2], slack = p.rows - nbox;
    for (int i = threadIdx.x; i < NPH * NCH * slack; i += kTcThreads) {
      const int pl = i / slack, row = nbox + i % slack;
      *(uint4*)(A + (size_t)pl * p.plane_bytes + (size_t)row * 16) = make_uint4(0, 0, 0, 0);
    }
  }
  fence_proxy_async_smem();
  bool ok = __syncthreads_and(mbar_wait_bounded(&bars[0], 0, kTcWaitNs));
  bool loads_done = ok, mma_done = true;

  const unsigned idesc = umma_idesc(p.N);
  const int tpg = kTmemCols / p.N;  // M-tiles per accumulator group
  const int n0 = slice * p.N;
  // Descriptor bases; per MMA only the start-address field (bits 0-13, in
  // 16-byte units) changes, by a whole number of rows / weight blocks, so the
  // issuing lanes add offsets to the 64-bit descriptors (shared addresses
  // stay below 2^18 bytes, so the field never carries).
  const unsigned long long da0 = umma_desc(smem_u32(A), (unsigned)p.plane_bytes, 128u);
  const unsigned long long db0 = umma_desc(smem_u32(W), (unsigned)(p.N >> 3) * 128u, 128u);
  const unsigned plane16 = (unsigned)p.plane_bytes >> 4;
  const unsigned wtap16 = (unsigned)(CIN * p.N * 2) >> 4, wk16 = (unsigned)(p.N >> 3) * 8u;
  // row offset (16-byte units, including the plane of stride-2 taps) of every tap
  int toff[27];
#pragma unroll
  for (int k = 0; k < 27; k++) {
    const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    int off, plane0;
    if (STRIDE == 2) {
      off = -(dx < 0) - HX * ((dy < 0) + HY * (dz < 0));
      plane0 = ((dx != 0) + 2 * (dy != 0) + 4 * (dz != 0)) * NCH;
    } else {
      off = dx + HX * (dy + HY * dz);
      plane0 = 0;
    }
    toff[k] = plane0 * (int)plane16 + off;
  }
  int phase = 0;
  for (int g0 = 0; g0 < p.tiles && ok; g0 += tpg) {
    const int g1 = min(p.tiles, g0 + tpg), ntg = g1 - g0;
    // Groups with fewer tiles than warps split the taps of a tile over S
    // warps, each into its own accumulator columns (summed in the
    // epilogue), so every warp issues MMAs.
    int S = 1;
    while (S * 2 * ntg <= NWARP && S * 2 * ntg * p.N <= kTmemCols) S *= 2;
    if (lane == 0) {
      tc_fence_after();
      if (S == 1) {
        // every warp's lane 0 issues the MMAs of its tiles (t = g0 + warp + 4j)
        for (int t = g0 + warp; t < g1; t += NWARP) {
          const unsigned d = tmem + (unsigned)((t - g0) * p.N);
          const unsigned long long dat = da0 + (unsigned)(p.q0 + 128 * t);
#pragma unroll
          for (int k = 0; k < 27; k++) {
            const unsigned long long dak = dat + (unsigned long long)(long long)toff[k];
            const unsigned long long dbk = db0 + (unsigned long long)k * wtap16;
#pragma unroll
            for (int j = 0; j < KSTEPS; j++)
              umma(d, dak + (unsigned long long)(2 * j) * plane16, dbk + (unsigned long long)(2 * j) * wk16, idesc,
                   (k | j) != 0);
          }
        }
      } else if (warp < ntg * S) {
        // warp = (tile, split): taps k = split, split + S, ...
        const int t = g0 + warp / S, sp = warp % S;
        const unsigned d = tmem + (unsigned)(((t - g0) * S + sp) * p.N);
        const unsigned long long dat = da0 + (unsigned)(p.q0 + 128 * t);
        for (int k = sp; k < 27; k += S) {
          const unsigned long long dak = dat + (unsigned long long)(long long)toff[k];
          const unsigned long long dbk = db0 + (unsigned long long)k * wtap16;
#pragma unroll
          for (int j = 0; j < KSTEPS; j++)
            umma(d, dak + (unsigned long long)(2 * j) * plane16, dbk + (unsigned long long)(2 * j) * wk16, idesc,
                 (k != sp || j != 0) ? 1u : 0u);
        }
      }
      umma_commit(&bars[1 + warp]);
    }
    __syncwarp();
    bool w_ok = true;
    for (int w = 0; w < NWARP; w++) w_ok = w_ok && mbar_wait_bounded(&bars[1 + w], phase, kTcWaitNs);
    ok = __syncthreads_and(w_ok);
    phase ^= 1;
    tc_fence_after();
    if (!ok) {
      mma_done = false;
      break;
    }
    // epilogue: thread = one row of each tile of the group
    for (int t = g0; t < g1; t++) {
      const int prow = p.q0 + 128 * t + 32 * warp + lane;
      const int hz = prow / (HX * HY), rem = prow - hz * HX * HY;
      const int hy = rem / HX, hx = rem - hy * HX;
      const int X = x0 + hx - 1, Y = y0 + hy - 1, Z = z0 + hz - 1;
      const bool valid = hx >= 1 && hx <= p.brick[0] && hy >= 1 && hy <= p.brick[1] && hz >= 1 &&
                         hz <= p.brick[2] && X < p.dims[0] && Y < p.dims[1] && Z < p.dims[2];
      const long long v = X + (long long)p.dims[0] * (Y + (long long)p.dims[1] * Z);
      for (int c = 0; c < p.N; c += 16) {
        float acc[16];
        tmem_ld16(tmem + ((unsigned)(32 * warp) << 16) + (unsigned)((t - g0) * S * p.N + c), acc);
        for (int sp = 1; sp < S; sp++) {
          float part[16];
          tmem_ld16(tmem + ((unsigned)(32 * warp) << 16) + (unsigned)(((t - g0) * S + sp) * p.N + c), part);
#pragma unroll
          for (int i = 0; i < 16; i++) acc[i] += part[i];
        }
        if (!valid) continue;
        if (p.out_f32) {
          if (n0 + c == 0) p.out_f32[v] = acc[0] + sbias[0];
          continue;
        }
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
          float y = acc[i] + sbias[c + i];
          if (p.act && y < 0.f) y *= kLeaky;
          o[i] = __float2bfloat16(y);
        }
        uint4* dst = (uint4*)(p.out + v * p.cout + n0 + c);
        dst[0] = ((const uint4*)o)[0];
        dst[1] = ((const uint4*)o)[1];
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  if (!ok) {
    // a bounded wait gave up: report it, then give the copies and MMAs still
    // in flight one more bounded wait before the shared memory and the
    // accumulator columns are released
    if (threadIdx.x == 0) {
      if (p.err) atomicExch(p.err, 1);
      if (!loads_done) mbar_wait_bounded(&bars[0], 0, kTcWaitNs);
    }
    if (!mma_done && lane == 0) mbar_wait_bounded(&bars[1 + warp], phase ^ 1, kTcWaitNs);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---- the persistent, pipelined form ----
// CTA c serves output-channel slice c % nslices and loops over the bricks
// c / nslices, c / nslices + gridDim.x / nslices, ...  Three roles run at
// once:
// - warp 4 kEpiGroups (lane 0) brings a brick's halo in by TMA into one of astages
//   shared-memory stages (full[stage]);
// - the next warp (lane 0) issues the MMAs of one 128-row tile at a time into one
//   of nacc accumulators of N TMEM columns, commits each tile to
//   mdone[acc], and after a brick's last tile commits bfree[stage] (the
//   stage may be refilled once those MMAs have read it);
// - warps 0 .. 4 kEpiGroups - 1, groups of four taking tiles in turn, read each
//   finished accumulator back (warp w owns TMEM lanes 32 (w % 4) .. + 31,
//   those of its sub-partition), write the outputs and free it (afree[acc],
//   one arrival per warp of the group).  One group of four warps, one per
//   sub-partition, leaves every latency of the epilogue exposed; several
//   overlap.  Accumulator acc is read by group acc % kEpiGroups only.
// So the epilogue of a tile overlaps the MMAs of the next ones, and with two
// stages the copy of the next brick overlaps the MMAs of the current one.
// The slice's weights are loaded once per CTA.
//
// FOLD (stride 1): the MMAs of a tile are 9 (dy, dz) groups of K = cin, each
// against the three dx taps side by side (N = 3 nout columns, column
// (dx + 1) nout + c), so a 16-channel layer issues 9 MMAs of N = 48 per tile
// instead of 27 of N = 16.  The accumulator then holds D_dx[rho] =
// sum over (dy, dz) of A[rho + HX dy + HX HY dz] W[dx, dy, dz], and output
// row r is D_-1[r - 1] + D_0[r] + D_+1[r + 1]: the neighbouring rows come
// from the neighbouring lanes (shuffles), and across the warps' 32-row
// boundaries through shared memory.  A tile's 128 rows produce the 126
// outputs between its first and last row, so tiles step by 126 rows.
//
// Every wait is bounded; a role whose wait gives up sets *err, stops, and
// gives the copies or MMAs it has in flight one more bounded wait.
constexpr int kEpiGroups = 3;  // groups of four epilogue warps, alternate tiles
constexpr int kPipeThreads = 32 * (4 * kEpiGroups + 2);
constexpr int kPipeAcc = 4;  // most accumulators in the ring
static_assert(kPipeAcc >= kEpiGroups, "every epilogue group needs an accumulator");
constexpr int kPipeBars = 5 + 2 * kPipeAcc + 2 * kEpiGroups;
constexpr int kFoldChunks = 2;  // 16-channel chunks of a folded slice (nout <= 32)

__device__ __forceinline__ void mbar_arrive_cta(unsigned long long* m) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(m)) : "memory");
}
// Bias, activation and store of 16 output channels of one voxel.
__device__ __forceinline__ void store16(const ConvTcParams& p, long long v, int n0, int c, const float* sbias,
                                        const float (&acc)[16]) {
  if (p.out_f32) {
    if (n0 + c == 0) p.out_f32[v] = acc[0] + sbias[0];
    return;
  }
  __align__(16) __nv_bfloat16 o[16];
#pragma unroll
  for (int i = 0; i < 16; i++) {
    float y = acc[i] + sbias[c + i];
    if (p.act && y < 0.f) y *= kLeaky;
    o[i] = __float2bfloat16(y);
  }
  uint4* dst = (uint4*)(p.out + v * p.cout + n0 + c);
  dst[0] = ((const uint4*)o)[0];
  dst[1] = ((const uint4*)o)[1];
}

template <int CIN, int STRIDE, bool FOLD>
__global__ void __launch_bounds__(kPipeThreads) k_conv_pipe(const __grid_constant__ ConvTcParams p) {
  static_assert(!FOLD || STRIDE == 1, "the dx fold needs stride 1");
  constexpr int NCH = CIN / 8, KSTEPS = CIN / 16, NPH = STRIDE == 2 ? 8 : 1;
  constexpr int NG = FOLD ? 9 : 27;       // MMA groups per K step
  constexpr int TSTEP = FOLD ? 126 : 128;  // output rows per tile
  if (p.skip && *p.skip) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int nst = p.astages, nacc = p.nacc;
  const size_t stage_bytes = (size_t)NPH * NCH * p.plane_bytes;
  unsigned char* W = smem + (size_t)nst * stage_bytes;
  const unsigned wbytes = 27u * CIN * p.nout * 2u;
  // wbar, full[2], bfree[2], mdone[kPipeAcc], afree[kPipeAcc], xbar[kEpiGroups][2]
  unsigned long long* bars = (unsigned long long*)(W + wbytes);  // wbytes is a multiple of 16
  unsigned long long *wbar = bars, *full = bars + 1, *bfree = bars + 3, *mdone = bars + 5,
                     *afree = bars + 5 + kPipeAcc, *xbar = bars + 5 + 2 * kPipeAcc;
  unsigned* tmem_slot = (unsigned*)(bars + kPipeBars);
  float* sbias = (float*)(tmem_slot + 2);  // nout floats
  float* xs = sbias + p.nout;              // FOLD: [kEpiGroups][2][2][4][nout] edge rows
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int HX = p.halo[0], HY = p.halo[1];
  const int slice = blockIdx.x % p.nslices;
  const int cpos = blockIdx.x / p.nslices, cstride = gridDim.x / p.nslices;
  const int nbricks = p.nb[0] * p.nb[1] * p.nb[2];
  const int nunits = cpos < nbricks ? (nbricks - 1 - cpos) / cstride + 1 : 0;
  auto brick_origin = [&](int u, int& x0, int& y0, int& z0) {
    const int b = cpos + u * cstride;
    x0 = (b % p.nb[0]) * p.brick[0];
    y0 = ((b / p.nb[0]) % p.nb[1]) * p.brick[1];
    z0 = (b / (p.nb[0] * p.nb[1])) * p.brick[2];
  };

  if (threadIdx.x == 0) {
    mbar_init(wbar, 1);
    for (int i = 0; i < 2; i++) {
      mbar_init(full + i, 1);
      mbar_init(bfree + i, 1);
    }
    for (int i = 0; i < kPipeAcc; i++) {
      mbar_init(mdone + i, 1);
      mbar_init(afree + i, 4);
    }
    for (int i = 0; i < 2 * kEpiGroups; i++) mbar_init(xbar + i, 4);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(tmem_slot, (unsigned)p.acc_cols);
  for (int i = threadIdx.x; i < p.nout; i += blockDim.x) {
    const int co = slice * p.nout + i;
    sbias[i] = co < p.cout ? p.bias[co] : 0.f;
  }
  {
    // rows past the halo box that tap shifts of the last tiles read: zeros,
    // in every stage, once (the copies never write them)
    const int nbox = HX * HY * p.halo[2], slack = p.rows - nbox;
    const int per_stage = NPH * NCH * slack;
    for (int i = threadIdx.x; i < nst * per_stage; i += blockDim.x) {
      const int st = i / per_stage, rem = i % per_stage;
      const int pl = rem / slack, row = nbox + rem % slack;
      *(uint4*)(smem + st * stage_bytes + (size_t)pl * p.plane_bytes + (size_t)row * 16) = make_uint4(0, 0, 0, 0);
    }
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  const unsigned abytes = (unsigned)NPH * NCH * 16u * (unsigned)(HX * HY * p.halo[2]);
  const int ntiles = nunits * p.tiles;
  bool ok = true;

  if (warp == 4 * kEpiGroups) {
    if (lane == 0) {
      int issued = 0;
      mbar_expect_tx(wbar, wbytes);
      bulk_g2s(W, p.wpack + (size_t)slice * 27 * CIN * p.nout, wbytes, wbar);
      for (int u = 0; u < nunits; u++) {
        const int st = u % nst;
        if (u >= nst && !mbar_wait_bounded(bfree + st, (unsigned)((u / nst - 1) & 1), kTcWaitNs)) {
          ok = false;
          break;
        }
        int x0, y0, z0;
        brick_origin(u, x0, y0, z0);
        mbar_expect_tx(full + st, abytes);
        load_halo<NCH, STRIDE>(p, smem + st * stage_bytes, x0, y0, z0, full + st);
        issued = u + 1;
      }
      if (!ok) {
        if (p.err) atomicExch(p.err, 1);
        mbar_wait_bounded(wbar, 0, kTcWaitNs);
        for (int u = issued > nst ? issued - nst : 0; u < issued; u++)
          mbar_wait_bounded(full + u % nst, (unsigned)((u / nst) & 1), kTcWaitNs);
      }
    }
    __syncwarp();
  } else if (warp == 4 * kEpiGroups + 1) {
    if (lane == 0) {
      const unsigned idesc = umma_idesc(p.N);
      const unsigned long long db0 = umma_desc(smem_u32(W), (unsigned)(p.N >> 3) * 128u, 128u);
      const unsigned plane16 = (unsigned)p.plane_bytes >> 4;
      const unsigned wg16 = (unsigned)(CIN * p.N * 2) >> 4, wk16 = (unsigned)(p.N >> 3) * 8u;
      int toff[NG];
#pragma unroll
      for (int k = 0; k < NG; k++) {
        int off, plane0 = 0;
        if (FOLD) {
          const int dy = k % 3 - 1, dz = k / 3 - 1;
          off = HX * (dy + HY * dz);
        } else {
          const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
          if (STRIDE == 2) {
            off = -(dx < 0) - HX * ((dy < 0) + HY * (dz < 0));
            plane0 = ((dx != 0) + 2 * (dy != 0) + 4 * (dz != 0)) * NCH;
          } else {
            off = dx + HX * (dy + HY * dz);
          }
        }
        toff[k] = plane0 * (int)plane16 + off;
      }
      int g = 0;  // tiles issued
      ok = mbar_wait_bounded(wbar, 0, kTcWaitNs);
      for (int u = 0; u < nunits && ok; u++) {
        const int st = u % nst;
        if (!mbar_wait_bounded(full + st, (unsigned)((u / nst) & 1), kTcWaitNs)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const unsigned long long da0 = umma_desc(smem_u32(smem + st * stage_bytes), (unsigned)p.plane_bytes, 128u);
        for (int t = 0; t < p.tiles; t++, g++) {
          const int r = g % nacc;
          if (g >= nacc && !mbar_wait_bounded(afree + r, (unsigned)((g / nacc - 1) & 1), kTcWaitNs)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const unsigned d = tmem + (unsigned)(r * p.N);
          const unsigned long long dat = da0 + (unsigned)(p.q0 - (FOLD ? 1 : 0) + TSTEP * t);
#pragma unroll
          for (int k = 0; k < NG; k++) {
            const unsigned long long dak = dat + (unsigned long long)(long long)toff[k];
            const unsigned long long dbk = db0 + (unsigned long long)k * wg16;
#pragma unroll
            for (int j = 0; j < KSTEPS; j++)
              umma(d, dak + (unsigned long long)(2 * j) * plane16, dbk + (unsigned long long)(2 * j) * wk16, idesc,
                   (k | j) != 0);
          }
          umma_commit(mdone + r);
        }
        if (ok) umma_commit(bfree + st);
      }
      if (!ok) {
        if (p.err) atomicExch(p.err, 1);
        if (g > 0) mbar_wait_bounded(mdone + (g - 1) % nacc, (unsigned)(((g - 1) / nacc) & 1), kTcWaitNs);
      } else {
        // the last arrivals on bfree land before the CTA ends
        for (int u = nunits > nst ? nunits - nst : 0; u < nunits; u++)
          mbar_wait_bounded(bfree + u % nst, (unsigned)((u / nst) & 1), kTcWaitNs);
      }
    }
    __syncwarp();
  } else {
    // the epilogue: group eg takes tiles eg, eg + kEpiGroups, ...; its warp
    // q owns rows 32q .. 32q + 31 (TMEM lanes of the warp's sub-partition)
    const int n0 = slice * p.nout, eg = warp >> 2, q = warp & 3;
    const unsigned lanebase = tmem + ((unsigned)(32 * q) << 16);
    for (int g = eg; g < ntiles; g += kEpiGroups) {
      const int u = g / p.tiles, t = g - u * p.tiles, r = g % nacc, k = g / kEpiGroups;
      int x0, y0, z0;
      brick_origin(u, x0, y0, z0);
      // the MMA warp keeps going while the epilogue waits, so every lane
      // takes the same branch on the wait's outcome
      if (!__all_sync(0xffffffffu, mbar_wait_bounded(mdone + r, (unsigned)((g / nacc) & 1), kTcWaitNs))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int row = 32 * q + lane;
      const int prow = FOLD ? p.q0 - 1 + TSTEP * t + row : p.q0 + TSTEP * t + row;
      const int hz = prow / (HX * HY), rem = prow - hz * HX * HY;
      const int hy = rem / HX, hx = rem - hy * HX;
      const int X = x0 + hx - 1, Y = y0 + hy - 1, Z = z0 + hz - 1;
      const bool valid = (!FOLD || (row >= 1 && row <= 126)) && hx >= 1 && hx <= p.brick[0] && hy >= 1 &&
                         hy <= p.brick[1] && hz >= 1 && hz <= p.brick[2] && X < p.dims[0] && Y < p.dims[1] &&
                         Z < p.dims[2];
      const long long v = X + (long long)p.dims[0] * (Y + (long long)p.dims[1] * Z);
      const unsigned col0 = (unsigned)(r * p.N);
      if constexpr (FOLD) {
        // edge rows across the warps' boundaries: lane 31 posts D_-1 of its
        // row for the next warp's lane 0, lane 0 posts D_+1 for the previous
        // warp's lane 31.  The buffers and the mbarrier that publishes them
        // (one arrival per warp, a bounded wait) are the group's own and
        // alternate with its tiles (k counts them): a warp writes the buffers
        // of its tile k + 2 only after every warp of the group has arrived
        // for tile k + 1, that is after its reads of tile k.
        // All of the tile's columns are read with one wait (kFoldChunks x 16
        // output channels at most, checked by the plan).
        const int nout = p.nout, nch = nout / 16;
        float* xm = xs + (size_t)((eg * 2 + (k & 1)) * 2 + 0) * 4 * nout;
        float* xp = xs + (size_t)((eg * 2 + (k & 1)) * 2 + 1) * 4 * nout;
        unsigned raw[3][kFoldChunks][16];
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
          for (int h = 0; h < kFoldChunks; h++)
            if (h < nch) tmem_ld16_async(lanebase + col0 + (unsigned)(b * nout + 16 * h), raw[b][h]);
        tmem_wait_ld();
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
          for (int h = 0; h < kFoldChunks; h++) reg_pin16(raw[b][h]);
#pragma unroll
        for (int h = 0; h < kFoldChunks; h++) {
          if (h >= nch) break;
          if (lane == 31)
#pragma unroll
            for (int i = 0; i < 16; i++) xm[q * nout + 16 * h + i] = __uint_as_float(raw[0][h][i]);
          if (lane == 0)
#pragma unroll
            for (int i = 0; i < 16; i++) xp[q * nout + 16 * h + i] = __uint_as_float(raw[2][h][i]);
        }
        __syncwarp();
        unsigned long long* xb = xbar + 2 * eg + (k & 1);
        if (lane == 0) mbar_arrive_cta(xb);
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(xb, (unsigned)((k >> 1) & 1), kTcWaitNs))) {
          ok = false;
          break;
        }
#pragma unroll
        for (int h = 0; h < kFoldChunks; h++) {
          if (h >= nch) break;
          float acc[16];
#pragma unroll
          for (int i = 0; i < 16; i++) {
            float left = __shfl_up_sync(0xffffffffu, __uint_as_float(raw[0][h][i]), 1);
            float right = __shfl_down_sync(0xffffffffu, __uint_as_float(raw[2][h][i]), 1);
            if (lane == 0) left = q > 0 ? xm[(q - 1) * nout + 16 * h + i] : 0.f;
            if (lane == 31) right = q < 3 ? xp[(q + 1) * nout + 16 * h + i] : 0.f;
            acc[i] = (left + __uint_as_float(raw[1][h][i])) + right;
          }
          if (valid) store16(p, v, n0, 16 * h, sbias, acc);
        }
      } else {
        for (int c = 0; c < p.nout; c += 16) {
          float acc[16];
          tmem_ld16(lanebase + col0 + (unsigned)c, acc);
          if (valid) store16(p, v, n0, c, sbias, acc);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cta(afree + r);
    }
    if (!ok && lane == 0 && p.err) atomicExch(p.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, (unsigned)p.acc_cols);
  }
}

// wpack[slice][tap][kc][ng][n8][k8]: canonical K-major B blocks (8 output
// channels x 8 input channels, 16-byte rows) per tap and output-channel slice.
__global__ void k_pack_tc(const __nv_bfloat16* __restrict__ w, int cin, int cout, int N, int nslices,
                          __nv_bfloat16* wp) {
  const long long total = (long long)nslices * 27 * cin * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int k8 = (int)(i % 8);
    const int n8 = (int)((i / 8) % 8);
    const long long r = i / 64;
    const int ng = (int)(r % (N / 8));
    const int kc = (int)((r / (N / 8)) % (cin / 8));
    const int tap = (int)((r / ((N / 8) * (cin / 8))) % 27);
    const int slice = (int)(r / ((long long)(N / 8) * (cin / 8) * 27));
    const int ci = kc * 8 + k8, co = slice * N + ng * 8 + n8;
    wp[i] = co < cout ? w[((size_t)tap * cin + ci) * cout + co] : __float2bfloat16(0.f);
  }
}

// The dx-folded layout: wpack[slice][g][kc][ng][n8][k8] with g = (dy + 1) +
// 3 (dz + 1) and column n = ng 8 + n8 = (dx + 1) W + c over N = 3 W columns
// (W output channels per slice, channel slice W + c).
__global__ void k_pack_fold(const __nv_bfloat16* __restrict__ w, int cin, int cout, int W, int nslices,
                            __nv_bfloat16* wp) {
  const int N = 3 * W;
  const long long total = (long long)nslices * 9 * cin * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int k8 = (int)(i % 8);
    const int n8 = (int)((i / 8) % 8);
    const long long r = i / 64;
    const int ng = (int)(r % (N / 8));
    const int kc = (int)((r / (N / 8)) % (cin / 8));
    const int g = (int)((r / ((N / 8) * (cin / 8))) % 9);
    const int slice = (int)(r / ((long long)(N / 8) * (cin / 8) * 9));
    const int n = ng * 8 + n8, dxi = n / W, co = slice * W + n % W;
    const int tap = dxi + 3 * g, ci = kc * 8 + k8;
    wp[i] = co < cout ? w[((size_t)tap * cin + ci) * cout + co] : __float2bfloat16(0.f);
  }
}

int ceil_div(int a, int b) { return (a + b - 1) / b; }

// cuTensorMapEncodeTiled from the driver, found through the runtime (no link
// against libcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// The input's TMA descriptor: dims (cin, x, y, z) of the channels-last BF16
// input; box 8 channels x the halo brick, with a traversal stride of 2 along
// x, y, z for stride 2 (the box then spans 2 x halo voxels per axis and
// loads halo of them).  Returns false when a limit of the copy is not met.
bool encode_input_map(ConvTcParams& p) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  if (reinterpret_cast<uintptr_t>(p.in) % 16 != 0 || p.cin % 8 != 0) return false;
  const int s = p.stride;
  cuuint64_t gdim[4] = {(cuuint64_t)p.cin, (cuuint64_t)p.in_dims[0], (cuuint64_t)p.in_dims[1],
                        (cuuint64_t)p.in_dims[2]};
  cuuint64_t gstride[3] = {(cuuint64_t)p.cin * 2, (cuuint64_t)p.cin * 2 * p.in_dims[0],
                           (cuuint64_t)p.cin * 2 * p.in_dims[0] * p.in_dims[1]};
  cuuint32_t box[4] = {8, (cuuint32_t)(s * p.halo[0]), (cuuint32_t)(s * p.halo[1]), (cuuint32_t)(s * p.halo[2])};
  cuuint32_t estride[4] = {1, (cuuint32_t)s, (cuuint32_t)s, (cuuint32_t)s};
  for (int a = 1; a < 4; a++)
    if (box[a] < 1 || box[a] > 256) return false;
  const CUresult r = enc(&p.tmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(p.in), gdim,
                         gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

int conv_tc_slice_width(int cin, int cout, int stride) {
  // resident weights of a slice: up to 112 KiB next to a stride-1 brick, 56
  // KiB next to the eight phase planes of a stride-2 brick
  const long long cap = stride == 2 ? 56 * 1024 : 112 * 1024;
  int N = cout < 16 ? 16 : cout;
  while (N > 16 && 27LL * cin * N * 2 > cap) N /= 2;
  return N;
}

bool conv_tc_supported(const ConvDesc& d) {
  bool dims_ok = true;
  for (int a = 0; a < 3; a++)
    dims_ok = dims_ok && (d.stride == 1 ? d.in_dims[a] == d.out_dims[a] : d.in_dims[a] == 2 * d.out_dims[a] - 1);
  // The single-output last layer (FP32 output, no activation) runs as a
  // 16-column MMA whose first column is stored: the 15 unused columns cost
  // little next to the shared-memory reads of the A operand, which the
  // CUDA-core form of that layer is bound by.
  const bool last = d.cout == 1 && d.out_f32 && !d.out && !d.act;
  return (d.stride == 1 || d.stride == 2) && dims_ok && d.cb == 0 && (d.ca == 16 || d.ca == 32 || d.ca == 64) &&
         (d.cout == 16 || d.cout == 32 || d.cout == 64 || last);
}

cudaError_t conv_tc_pack(const __nv_bfloat16* w, int cin, int cout, int stride, __nv_bfloat16* wpack,
                         cudaStream_t s, int fold) {
  const int N = conv_tc_slice_width(cin, cout, stride);
  const int ns = ceil_div(cout < 16 ? 16 : cout, N);
  const long long total = (long long)ns * 27 * cin * N;
  if (fold) {
    if (stride != 1) return cudaErrorInvalidValue;
    k_pack_fold<<<(int)std::min<long long>((total + 255) / 256, 4096), 256, 0, s>>>(w, cin, cout, N, ns, wpack);
    return cudaGetLastError();
  }
  k_pack_tc<<<(int)std::min<long long>((total + 255) / 256, 4096), 256, 0, s>>>(w, cin, cout, N, ns, wpack);
  return cudaGetLastError();
}

long long conv_tc_pack_elems(int cin, int cout, int stride) {
  const int N = conv_tc_slice_width(cin, cout, stride);
  return (long long)ceil_div(cout < 16 ? 16 : cout, N) * 27 * cin * N;
}

namespace {

// Halo-brick layout of the persistent form for bricks tz voxels deep: rows
// per plane, tiles, shared memory per stage.  A tile computes rows
// [first, first + 127] of the halo box and outputs 128 of them (126 with the
// dx fold, whose first and last rows only feed their neighbours).
int pipe_tstep(const ConvTcParams& p) { return p.fold ? 126 : 128; }
void pipe_rows(const ConvTcParams& p, int& lo, int& hi) {
  // lowest and highest shared-memory row that an MMA of the brick reads
  const int HX = p.halo[0], HY = p.halo[1];
  const int first = p.fold ? p.q0 - 1 : p.q0, last = first + pipe_tstep(p) * (p.tiles - 1) + 127;
  const int down = p.fold ? HX + HX * HY : 1 + HX + HX * HY;
  const int up = p.fold ? HX + HX * HY : (p.stride == 2 ? 0 : 1 + HX + HX * HY);
  lo = first - down;
  hi = last + up;
}
void pipe_layout(ConvTcParams& p, int tz, int hpad) {
  const int HX = p.halo[0], HY = p.halo[1];
  p.brick[2] = tz;
  p.halo[2] = tz + hpad;
  p.q0 = 1 + HX + HX * HY;
  const int last = p.brick[0] + HX * (p.brick[1] + HY * p.brick[2]);
  p.tiles = ceil_div(last - p.q0 + 1, pipe_tstep(p));
  int lo, hi;
  pipe_rows(p, lo, hi);
  const int rows = std::max(HX * HY * p.halo[2], hi + 1);
  p.rows = (rows + 7) & ~7;
  p.plane_bytes = ((p.rows * 16) + 1023) & ~1023;
}

// The persistent form's bricks: the depth tz that minimises an estimate of
// the CTA's time.  A brick's MMAs take tiles x (cycles of a tile's MMAs,
// bound by the shared-memory reads of A and B at 128 bytes per clock), its
// halo copy (16-byte rows) about bytes / 16 cycles; with two stages the
// slower of the two sets the pace after the first copy, with one they add.
// Returns false when no depth fits.
bool plan_pipe(ConvTcParams& p, int num_sms, ConvTcPlan& plan) {
  const int nchunk = p.cin / 8, nphase = p.stride == 2 ? 8 : 1, hpad = p.stride == 2 ? 1 : 2;
  const long long wbytes = 27LL * p.cin * p.nout * 2;
  const long long extra = 8LL * kPipeBars + 8 + 4LL * p.nout + (p.fold ? kEpiGroups * 16LL * 4 * p.nout : 0);
  const long long cap = 227 * 1024;
  const int cps = std::max(1, num_sms / p.nslices);
  const double tile_cycles = (p.fold ? 9.0 : 27.0) * (p.cin / 16) * (32.0 + p.N / 4.0);
  double best = -1;
  int best_tz = 0, best_nst = 0;
  for (int tz = 1; tz <= p.dims[2]; tz++) {
    pipe_layout(p, tz, hpad);
    const long long stage = (long long)nphase * nchunk * p.plane_bytes;
    const int nbricks = p.nb[0] * p.nb[1] * ceil_div(p.dims[2], tz);
    const int per_cta = ceil_div(nbricks, cps);
    int nst = 0;
    if (per_cta > 1 && 2 * stage + wbytes + extra <= cap)
      nst = 2;
    else if (stage + wbytes + extra <= cap)
      nst = 1;
    if (!nst) break;  // deeper bricks only grow
    const double copy_cycles = (double)nphase * nchunk * 16.0 * p.halo[0] * p.halo[1] * p.halo[2] / 16.0;
    const double mma_cycles = (double)p.tiles * tile_cycles;
    const double cost = nst == 2 ? copy_cycles + per_cta * std::max(mma_cycles, copy_cycles)
                                 : per_cta * (mma_cycles + copy_cycles);
    if (best < 0 || cost <= best) {
      best = cost;
      best_tz = tz;
      best_nst = nst;
    }
  }
  if (!best_tz) return false;
  pipe_layout(p, best_tz, hpad);
  p.astages = best_nst;
  // accumulator ring: a multiple of the epilogue groups, so that every
  // accumulator is read by one group only (a group waits on each phase of
  // its accumulators' mdone in turn; an mbarrier parity wait cannot look two
  // phases ahead), within 256 TMEM columns where it can (two CTAs per SM)
  const int per_group = std::max(1, std::min(256 / (kEpiGroups * p.N), kPipeAcc / kEpiGroups));
  p.nacc = kEpiGroups * per_group;
  int cols = 32;
  while (cols < p.nacc * p.N) cols *= 2;
  p.acc_cols = cols;
  plan.smem = (size_t)best_nst * nphase * nchunk * p.plane_bytes + wbytes + extra;
  const int nbricks = p.nb[0] * p.nb[1] * ceil_div(p.dims[2], best_tz);
  plan.grid_x = p.nslices * std::min(nbricks, cps);
  plan.pipe = 1;
  return true;
}

}  // namespace

int conv_tc_plan(const ConvDesc& d, const __nv_bfloat16* wpack, int num_sms, ConvTcPlan& plan, int pipe) {
  std::memset(&plan, 0, sizeof(plan));
  if (!conv_tc_supported(d)) return -1;
  ConvTcParams& p = plan.p;
  for (int a = 0; a < 3; a++) {
    p.dims[a] = d.out_dims[a];
    p.in_dims[a] = d.in_dims[a];
  }
  p.in = d.inA;
  p.stride = d.stride;
  p.cin = d.ca;
  p.cout = d.cout;
  p.N = conv_tc_slice_width(d.ca, d.cout, d.stride);
  p.nslices = ceil_div(d.cout < 16 ? 16 : d.cout, p.N);
  p.nout = p.N;
  if (pipe == 2) {
    if (d.stride != 1) return -1;
    p.fold = 1;
    p.N = 3 * p.nout;
  }
  const int nchunk = p.cin / 8, nphase = d.stride == 2 ? 8 : 1, hpad = d.stride == 2 ? 1 : 2;
  const long long wbytes = 27LL * p.cin * p.N * 2;
  for (int a = 0; a < 2; a++) {
    p.nb[a] = ceil_div(p.dims[a], 16);
    p.brick[a] = ceil_div(p.dims[a], p.nb[a]);
    p.halo[a] = p.brick[a] + hpad;
  }
  if (pipe) {
    if (!plan_pipe(p, num_sms, plan)) return -3;
  }
  // bricks along z: one wave of two CTAs per SM when two fit next to each
  // other in shared memory, else one wave of one CTA per SM with deeper bricks
  for (int per_sm = 2; per_sm >= 1 && !pipe; per_sm--) {
    const long long budget = per_sm == 2 ? 113 * 1024 : 220 * 1024;
    const int target = std::max(1, per_sm * num_sms / (p.nb[0] * p.nb[1] * p.nslices));
    int tz = std::max(1, ceil_div(p.dims[2], target));
    for (;; tz--) {
      p.brick[2] = tz;
      p.halo[2] = tz + hpad;
      const int HX = p.halo[0], HY = p.halo[1];
      p.q0 = 1 + HX + HX * HY;
      const int last = p.brick[0] + HX * (p.brick[1] + HY * p.brick[2]);
      p.tiles = ceil_div(last - p.q0 + 1, 128);
      const int off_max = d.stride == 2 ? 0 : 1 + HX + HX * HY;
      int rows = std::max(HX * HY * p.halo[2], p.q0 + 128 * p.tiles + off_max);
      p.rows = (rows + 7) & ~7;
      p.plane_bytes = ((p.rows * 16) + 1023) & ~1023;
      plan.smem = (size_t)nphase * nchunk * p.plane_bytes + wbytes + 64 + 4 * p.N;
      if ((long long)plan.smem <= budget || tz == 1) break;
    }
    const int ctas = p.nb[0] * p.nb[1] * ceil_div(p.dims[2], p.brick[2]) * p.nslices;
    if ((long long)plan.smem <= budget && ctas <= per_sm * num_sms) break;  // fits one wave
  }
  if (plan.smem > 227 * 1024) return -3;
  {
    // every shared-memory row the MMAs address lies inside its plane, the
    // halo box stays small, and a group of tiles (the persistent form: the
    // accumulator ring) fits the TMEM columns
    const int HX = p.halo[0], HY = p.halo[1];
    const int off_min = 1 + HX + HX * HY, off_max = d.stride == 2 ? 0 : off_min;
    int lo = p.q0 - off_min, hi = p.q0 + 128 * p.tiles - 1 + off_max;
    if (pipe) pipe_rows(p, lo, hi);
    if (lo < 0 || hi >= p.rows || p.rows * 16 > p.plane_bytes || p.halo[0] > 256 || p.halo[1] > 256 ||
        p.halo[2] > 256 || p.tiles < 1 || p.N % 16 != 0 || p.N < 16 || p.cin % 16 != 0 || p.nout % 16 != 0 ||
        (!pipe && p.N > kTmemCols) ||
        (pipe && (p.N > 256 || p.nacc < 1 || p.nacc > kPipeAcc || p.nacc % kEpiGroups != 0 ||
                  p.nacc * p.N > p.acc_cols || p.acc_cols > 512 ||
                  plan.grid_x % p.nslices != 0 || (p.fold && p.nout > 16 * kFoldChunks))))
      return -5;
  }
  p.nb[2] = ceil_div(p.dims[2], p.brick[2]);
  if (!encode_input_map(p)) return -6;
  p.wpack = wpack;
  p.bias = d.bias;
  p.out = d.out;
  p.out_f32 = d.out_f32;
  p.act = d.act;
  p.skip = d.skip;
  if (!pipe) plan.grid_x = p.nb[0] * p.nb[1] * p.nb[2];
  plan.ready = 1;
  return 0;
}

cudaError_t conv3_forward_tc(const ConvTcPlan& plan, float* out_f32, const int* skip, int* err, cudaStream_t s) {
  ConvTcParams p = plan.p;
  if (p.out_f32 && out_f32) p.out_f32 = out_f32;
  p.skip = skip;
  p.err = err;
  void (*k)(ConvTcParams) = nullptr;
  if (plan.pipe) {
    switch (p.cin * 8 + p.stride * 2 + p.fold) {
      case 16 * 8 + 2: k = k_conv_pipe<16, 1, false>; break;
      case 16 * 8 + 3: k = k_conv_pipe<16, 1, true>; break;
      case 16 * 8 + 4: k = k_conv_pipe<16, 2, false>; break;
      case 32 * 8 + 2: k = k_conv_pipe<32, 1, false>; break;
      case 32 * 8 + 3: k = k_conv_pipe<32, 1, true>; break;
      case 32 * 8 + 4: k = k_conv_pipe<32, 2, false>; break;
      case 64 * 8 + 2: k = k_conv_pipe<64, 1, false>; break;
      case 64 * 8 + 3: k = k_conv_pipe<64, 1, true>; break;
      case 64 * 8 + 4: k = k_conv_pipe<64, 2, false>; break;
      default: return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    k<<<plan.grid_x, kPipeThreads, plan.smem, s>>>(p);
    return cudaGetLastError();
  }
  switch (p.cin * 4 + p.stride) {
    case 16 * 4 + 1: k = k_conv_tc<16, 1>; break;
    case 16 * 4 + 2: k = k_conv_tc<16, 2>; break;
    case 32 * 4 + 1: k = k_conv_tc<32, 1>; break;
    case 32 * 4 + 2: k = k_conv_tc<32, 2>; break;
    case 64 * 4 + 1: k = k_conv_tc<64, 1>; break;
    case 64 * 4 + 2: k = k_conv_tc<64, 2>; break;
    default: return cudaErrorInvalidValue;
  }
  // The limit is a property of the kernel, not of the launch: layers of one
  // instantiation need different amounts, and a launch recorded in a CUDA
  // graph must stay valid after a later layer's launch, so the limit is
  // always the largest a block may have.
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  if (e != cudaSuccess) return e;
  k<<<dim3(plan.grid_x, p.nslices), kTcThreads, plan.smem, s>>>(p);
  return cudaGetLastError();
}

}  // namespace cfd
