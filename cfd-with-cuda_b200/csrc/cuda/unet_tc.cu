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
#include "unet.h"

namespace cfd {

namespace {

constexpr int kTcThreads = 128;
constexpr int kTmemCols = 128;
constexpr unsigned long long kTcWaitNs = 2000000000ULL;

struct Dims6 {
  int c[3], f[3];
};

__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
  // SWIZZLE_NONE, K-major canonical layout: 8-row core matrices of 16-byte
  // rows; lbo = byte distance between the two K halves, sbo = between 8-row
  // groups; version field (bits 46-47) = 1.
  unsigned long long d = (unsigned long long)((saddr >> 4) & 0x3FFFu);
  d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ULL << 46;
  return d;
}

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

__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_alloc(unsigned* slot, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
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
                         cudaStream_t s) {
  const int N = conv_tc_slice_width(cin, cout, stride);
  const int ns = ceil_div(cout < 16 ? 16 : cout, N);
  const long long total = (long long)ns * 27 * cin * N;
  k_pack_tc<<<(int)std::min<long long>((total + 255) / 256, 4096), 256, 0, s>>>(w, cin, cout, N, ns, wpack);
  return cudaGetLastError();
}

long long conv_tc_pack_elems(int cin, int cout, int stride) {
  const int N = conv_tc_slice_width(cin, cout, stride);
  return (long long)ceil_div(cout < 16 ? 16 : cout, N) * 27 * cin * N;
}

int conv_tc_plan(const ConvDesc& d, const __nv_bfloat16* wpack, int num_sms, ConvTcPlan& plan) {
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
  const int nchunk = p.cin / 8, nphase = d.stride == 2 ? 8 : 1, hpad = d.stride == 2 ? 1 : 2;
  const long long wbytes = 27LL * p.cin * p.N * 2;
  for (int a = 0; a < 2; a++) {
    p.nb[a] = ceil_div(p.dims[a], 16);
    p.brick[a] = ceil_div(p.dims[a], p.nb[a]);
    p.halo[a] = p.brick[a] + hpad;
  }
  // bricks along z: one wave of two CTAs per SM when two fit next to each
  // other in shared memory, else one wave of one CTA per SM with deeper bricks
  for (int per_sm = 2; per_sm >= 1; per_sm--) {
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
    // halo box stays small, and a group of tiles fits the TMEM columns
    const int HX = p.halo[0], HY = p.halo[1];
    const int off_min = 1 + HX + HX * HY, off_max = d.stride == 2 ? 0 : off_min;
    if (p.q0 - off_min < 0 || p.q0 + 128 * p.tiles - 1 + off_max >= p.rows || p.rows * 16 > p.plane_bytes ||
        p.halo[0] > 256 || p.halo[1] > 256 || p.halo[2] > 256 || p.tiles < 1 || p.N > kTmemCols ||
        p.N % 16 != 0 || p.cin % 16 != 0)
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
  plan.grid_x = p.nb[0] * p.nb[1] * p.nb[2];
  plan.ready = 1;
  return 0;
}

cudaError_t conv3_forward_tc(const ConvTcPlan& plan, float* out_f32, const int* skip, int* err, cudaStream_t s) {
  ConvTcParams p = plan.p;
  if (p.out_f32 && out_f32) p.out_f32 = out_f32;
  p.skip = skip;
  p.err = err;
  void (*k)(ConvTcParams) = nullptr;
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
