// Tensor-core (tcgen05) 3x3x3 convolution, stride 1, for the U-Net's
// inference path.
//
// Implicit GEMM without an im2col buffer.  A CTA owns a brick of output
// voxels; TMA brings the brick plus a one-voxel halo into shared memory, one
// plane per 8 input channels, each halo voxel one 16-byte row of the plane
// (rows numbered hx + HX (hy + HY hz) over the halo box, zero-filled outside
// the grid).  In that numbering every tap (dx, dy, dz) is a constant row
// shift, so the A operand of tap k for 128 consecutive rows is the plane
// itself at a shifted start address: no data is copied per tap.  Rows that
// fall on the halo ring compute garbage that is never stored.  The weights of
// all 27 taps for the CTA's slice of output channels are resident in shared
// memory, pre-packed in the tensor core's canonical K-major layout.
//
// Stride 2 (the U-Net's down-sampling layers) runs on the same machinery
// after a space-to-depth pass splits the fine input into its 8 parity phases
// (voxel (2i+px, 2j+py, 2k+pz) -> phase px + 2py + 4pz at (i, j, k)): tap d
// of output X reads phase (d != 0) at coarse index X + (d == -1 ? -1 : 0),
// again a constant row shift inside that phase's planes (low-side halo only).
//
// One thread issues tcgen05.mma (M = 128 rows, N = output channels of the
// slice, K = 16 input channels) into a 128-column TMEM accumulator; the four
// warps read it back with tcgen05.ld (warp w owns rows 32w..32w+31), add the
// bias, apply the activation and store BF16 (or FP32) channels-last.
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

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}

__global__ void __launch_bounds__(kTcThreads) k_conv_tc(const __grid_constant__ CUtensorMap tmap, ConvTcParams p) {
  if (p.skip && *p.skip) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int nchunk = p.cin >> 3, nphase = p.stride == 2 ? 8 : 1;
  unsigned char* A = smem;
  unsigned char* W = smem + (size_t)nphase * nchunk * p.plane_bytes;
  const unsigned wbytes = 27u * p.cin * p.N * 2u;
  unsigned long long* bars = (unsigned long long*)(W + wbytes);  // wbytes is a multiple of 16
  unsigned* tmem_slot = (unsigned*)(bars + 2);

  const int b = blockIdx.x, slice = blockIdx.y;
  const int bx = b % p.nb[0], by = (b / p.nb[0]) % p.nb[1], bz = b / (p.nb[0] * p.nb[1]);
  const int x0 = bx * p.brick[0], y0 = by * p.brick[1], z0 = bz * p.brick[2];
  const int HX = p.halo[0], HY = p.halo[1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  float* sbias = (float*)(tmem_slot + 4);  // N floats
  for (int i = threadIdx.x; i < p.N; i += blockDim.x) {
    const int co = slice * p.N + i;
    sbias[i] = co < p.cout ? p.bias[co] : 0.f;
  }

  if (threadIdx.x == 0) {
    const unsigned box = (unsigned)(p.halo[0] * p.halo[1] * p.halo[2]) * 16u;
    mbar_expect_tx(&bars[0], nphase * nchunk * box + wbytes);
    for (int ph = 0; ph < nphase; ph++)
      for (int c = 0; c < nchunk; c++)
        tma_load_5d(A + (size_t)(ph * nchunk + c) * p.plane_bytes, &tmap, c * 8, x0 - 1, y0 - 1, z0 - 1, ph,
                    &bars[0]);
    bulk_g2s(W, p.wpack + (size_t)slice * 27 * p.cin * p.N, wbytes, &bars[0]);
  }
  bool ok = __syncthreads_and(mbar_wait_bounded(&bars[0], 0, kTcWaitNs));
  bool loads_done = ok, mma_done = true;

  const unsigned idesc = umma_idesc(p.N);
  const int tpg = kTmemCols / p.N;  // M-tiles per accumulator group
  const int ksteps = p.cin >> 4;
  const int n0 = slice * p.N;
  // Descriptor bases; per MMA only the start-address field (bits 0-13, in
  // 16-byte units) changes, by a whole number of rows / weight blocks, so the
  // issuing thread adds offsets to the 64-bit descriptors (shared addresses
  // stay below 2^18 bytes, so the field never carries).
  const unsigned long long da0 = umma_desc(smem_u32(A), (unsigned)p.plane_bytes, 128u);
  const unsigned long long db0 = umma_desc(smem_u32(W), (unsigned)(p.N >> 3) * 128u, 128u);
  const unsigned plane16 = (unsigned)p.plane_bytes >> 4;
  const unsigned wtap16 = (unsigned)(p.cin * p.N * 2) >> 4, wk16 = (unsigned)(p.N >> 3) * 8u;
  int phase = 0;
  for (int g0 = 0; g0 < p.tiles && ok; g0 += tpg) {
    const int g1 = min(p.tiles, g0 + tpg);
    if (threadIdx.x == 0) {
      tc_fence_after();
      // row offset (16-byte units, including the plane of stride-2 taps) of
      // every tap
      int toff[27];
#pragma unroll
      for (int k = 0; k < 27; k++) {
        const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
        int off, plane0;
        if (p.stride == 2) {
          off = -(dx < 0) - HX * ((dy < 0) + HY * (dz < 0));
          plane0 = ((dx != 0) + 2 * (dy != 0) + 4 * (dz != 0)) * nchunk;
        } else {
          off = dx + HX * (dy + HY * dz);
          plane0 = 0;
        }
        toff[k] = plane0 * (int)plane16 + off;
      }
      for (int t = g0; t < g1; t++) {
        const unsigned d = tmem + (unsigned)((t - g0) * p.N);
        const unsigned long long dat = da0 + (unsigned)(p.q0 + 128 * t);
        unsigned acc = 0;
#pragma unroll
        for (int k = 0; k < 27; k++) {
          const unsigned long long dak = dat + (unsigned long long)(long long)toff[k];
          const unsigned long long dbk = db0 + (unsigned long long)k * wtap16;
          for (int j = 0; j < ksteps; j++) {
            umma(d, dak + (unsigned long long)(2 * j) * plane16, dbk + (unsigned long long)(2 * j) * wk16, idesc,
                 acc);
            acc = 1;
          }
        }
      }
      umma_commit(&bars[1]);
    }
    ok = __syncthreads_and(mbar_wait_bounded(&bars[1], phase, kTcWaitNs));
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
        tmem_ld16(tmem + ((unsigned)(32 * warp) << 16) + (unsigned)((t - g0) * p.N + c), acc);
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
      if (!mma_done) mbar_wait_bounded(&bars[1], phase ^ 1, kTcWaitNs);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ph[phase][k][j][i][c] = in[2i+px][2j+py][2k+pz][c] (zero outside the fine
// grid), phase = px + 2py + 4pz, coarse dims cd; one thread per 8 channels.
__global__ void k_space_to_depth(const __nv_bfloat16* __restrict__ in, Dims6 g, int ch, __nv_bfloat16* ph,
                                 const int* skip) {
  if (skip && *skip) return;
  const int nc = ch / 8;
  const long long per = (long long)g.c[0] * g.c[1] * g.c[2];
  const long long total = 8 * per * nc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % nc);
    const long long v = (i / nc) % per;
    const int phs = (int)(i / (nc * per));
    const int x = (int)(v % g.c[0]), y = (int)((v / g.c[0]) % g.c[1]), z = (int)(v / ((long long)g.c[0] * g.c[1]));
    const int fx = 2 * x + (phs & 1), fy = 2 * y + ((phs >> 1) & 1), fz = 2 * z + (phs >> 2);
    uint4 val = make_uint4(0, 0, 0, 0);
    if (fx < g.f[0] && fy < g.f[1] && fz < g.f[2])
      val = *(const uint4*)(in + ((fx + (long long)g.f[0] * (fy + (long long)g.f[1] * fz)) * ch + 8 * c));
    *(uint4*)(ph + ((phs * per + v) * ch + 8 * c)) = val;
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

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiled)p;
  }
  return fn;
}

int ceil_div(int a, int b) { return (a + b - 1) / b; }

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
  return (d.stride == 1 || d.stride == 2) && dims_ok && d.cb == 0 && (d.ca == 16 || d.ca == 32 || d.ca == 64) &&
         (d.cout == 16 || d.cout == 32 || d.cout == 64 || (d.cout == 1 && d.out_f32 && !d.out));
}

long long conv_tc_phase_elems(const ConvDesc& d) {
  return d.stride == 2 ? 8LL * d.out_dims[0] * d.out_dims[1] * d.out_dims[2] * d.ca : 0;
}

cudaError_t conv_tc_space_to_depth(const ConvDesc& d, __nv_bfloat16* phase, const int* skip, cudaStream_t s) {
  Dims6 g;
  for (int a = 0; a < 3; a++) {
    g.c[a] = d.out_dims[a];
    g.f[a] = d.in_dims[a];
  }
  const long long total = conv_tc_phase_elems(d) / 8;
  k_space_to_depth<<<(int)std::min<long long>((total + 255) / 256, 148 * 16), 256, 0, s>>>(d.inA, g, d.ca, phase,
                                                                                           skip);
  return cudaGetLastError();
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

int conv_tc_plan(const ConvDesc& d, const __nv_bfloat16* wpack, const __nv_bfloat16* phase, int num_sms,
                 ConvTcPlan& plan) {
  std::memset(&plan, 0, sizeof(plan));
  if (!conv_tc_supported(d)) return -1;
  if (d.stride == 2 && !phase) return -1;
  EncodeTiled enc = encoder();
  if (!enc) return -2;
  ConvTcParams& p = plan.p;
  for (int a = 0; a < 3; a++) p.dims[a] = d.out_dims[a];
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
  // bricks along z: enough CTAs for two per SM, within the shared-memory budget
  const long long budget = 200 * 1024;
  const int target = ceil_div(2 * num_sms, p.nb[0] * p.nb[1] * p.nslices);
  int tz = std::max(1, ceil_div(p.dims[2], std::max(1, target)));
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
  if (plan.smem > 227 * 1024) return -3;
  {
    // every shared-memory row the MMAs address lies inside its plane, every
    // TMA box dimension is legal, and a group of tiles fits the TMEM columns
    const int HX = p.halo[0], HY = p.halo[1];
    const int off_min = 1 + HX + HX * HY, off_max = d.stride == 2 ? 0 : off_min;
    if (p.q0 - off_min < 0 || p.q0 + 128 * p.tiles - 1 + off_max >= p.rows || p.rows * 16 > p.plane_bytes ||
        p.halo[0] > 256 || p.halo[1] > 256 || p.halo[2] > 256 || p.tiles < 1 || p.N > kTmemCols ||
        p.N % 16 != 0 || p.cin % 16 != 0)
      return -5;
  }
  p.nb[2] = ceil_div(p.dims[2], p.brick[2]);
  p.wpack = wpack;
  p.bias = d.bias;
  p.out = d.out;
  p.out_f32 = d.out_f32;
  p.act = d.act;
  p.skip = d.skip;
  plan.grid_x = p.nb[0] * p.nb[1] * p.nb[2];
  // input [phase][Z][Y][X][C] BF16 (one phase for stride 1: the tensor
  // itself; eight coarse-grid phases for stride 2); box = one 8-channel chunk
  // of the halo brick of one phase
  const cuuint64_t vox = (cuuint64_t)p.dims[0] * p.dims[1] * p.dims[2];
  cuuint64_t gdim[5] = {(cuuint64_t)p.cin, (cuuint64_t)p.dims[0], (cuuint64_t)p.dims[1], (cuuint64_t)p.dims[2],
                        (cuuint64_t)nphase};
  cuuint64_t gstride[4] = {(cuuint64_t)p.cin * 2, (cuuint64_t)p.cin * 2 * p.dims[0],
                           (cuuint64_t)p.cin * 2 * p.dims[0] * p.dims[1], (cuuint64_t)p.cin * 2 * vox};
  cuuint32_t box[5] = {8, (cuuint32_t)p.halo[0], (cuuint32_t)p.halo[1], (cuuint32_t)p.halo[2], 1};
  cuuint32_t estride[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(&plan.tmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)(d.stride == 2 ? phase : d.inA), gdim,
                   gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return -4;
  plan.ready = 1;
  return 0;
}

cudaError_t conv3_forward_tc(const ConvTcPlan& plan, float* out_f32, const int* skip, int* err, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem);
  if (e != cudaSuccess) return e;
  ConvTcParams p = plan.p;
  if (p.out_f32 && out_f32) p.out_f32 = out_f32;
  p.skip = skip;
  p.err = err;
  k_conv_tc<<<dim3(plan.grid_x, p.nslices), kTcThreads, plan.smem, s>>>(plan.tmap, p);
  return cudaGetLastError();
}

}  // namespace cfd
