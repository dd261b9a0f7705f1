// Tensor-core form of the convection right-hand side in mixed precision:
// R1 = -A(Un) UnpHalf_prev (calculateMatrixA, blascoCodinaHuerta.cpp:3520-3685;
// calcAndAssembleMatrixA, CUDAcodes.cu:695-899), the factored sums of
// k_convect (convect.cu) with its two per-element contractions batched over
// 16 elements and issued as tcgen05.mma (kind::tf32, FP32 accumulators in
// tensor memory):
//
//   (1) Gauss-point values: rows (element e, quantity q) of the gathered
//       nodal data -- q = 0..2 the components of Un, q = 3..5 those of
//       UnpHalf_prev, q = 6, 7 zero -- times the basis table of the 8 Gauss
//       points {Sv, dSv/dxi, dSv/deta, dSv/dzeta}: M = 128 (16 elements x 8
//       rows), N = 32 (4 tables x 8 Gauss points), K = 27 nodes (padded to
//       32, four K-steps of 8).  Row (e, q) column (s, k) holds
//       u0_k^q (s = 0, q < 3) and d uprev^(q-3) / d xi_(s-1) at k (q >= 3);
//   (2) the weighted convective products c_k^d = (u0_k . grad uprev^d(k))
//       detJ_k w_k, formed per (element, Gauss point) on the CUDA cores from
//       (1) and the Jacobian of the 8-corner map, times Sv: M = 128 (rows
//       (e, d), d < 3), N = 32 (27 nodes), K = 8 Gauss points.
//
// TF32 keeps 10 of FP32's 23 mantissa bits.  Every operand is split as
// x = hi + lo (hi: x with its low 13 mantissa bits cleared, lo = x - hi,
// exact) and each product is accumulated as hi*hi + hi*lo + lo*hi, three MMAs
// into one accumulator; the dropped lo*lo term and the truncation of lo keep
// the sums within about 2^-21 of their magnitude.
//
// Operands sit in shared memory in the K-major, no-swizzle canonical layout
// of 8-row core matrices with 16-byte rows: per K-step of 8 values a tile of
// R rows is [K-half 0: R rows x 16 B][K-half 1: R rows x 16 B] (leading
// byte offset R x 16, stride byte offset 128).  One thread issues the MMAs of
// a tile and commits them to an mbarrier; all waits are bounded (a wait that
// gives up sets *err and the block leaves after one more bounded wait).  The
// scatter is one 16-byte FP32 vector reduction per element node, as in
// k_convect's mixed-precision path.  NGP = 8, no element colouring.
#include "kernels.h"
#include "tcgen05.cuh"

namespace cfd {

namespace {

constexpr int kCtThreads = 128;  // four warps: warp w owns TMEM lanes 32w..32w+31
constexpr int kCtElems = 16;     // elements per tile (M = 128 rows of 8)
constexpr int kCtCols = 64;      // TMEM columns: (1) in 0..31, (2) in 32..63
constexpr unsigned long long kCtWaitNs = 2000000000ULL;

// shared-memory carve-up (bytes; the MMA operand tiles first, 1024-aligned)
constexpr unsigned kA1 = 4 * 4096;  // 4 K-steps x 128 rows x 32 B
constexpr unsigned kB1 = 4 * 1024;  // 4 K-steps x 32 rows x 32 B
constexpr unsigned kA2 = 4096, kB2 = 1024;
constexpr unsigned oA1h = 0, oA1l = oA1h + kA1, oB1h = oA1l + kA1, oB1l = oB1h + kB1;
constexpr unsigned oA2h = oB1l + kB1, oA2l = oA2h + kA2, oB2h = oA2l + kA2, oB2l = oB2h + kB2;
constexpr int kSld = 33;                                    // row stride (floats) of the TMEM staging
constexpr unsigned oS = oB2l + kB2;                         // float[128][33]
// the gathered nodal values, float4[16][27] of Un then of uprev, share the
// staging area: they are dead once operand (1) is written, and the staging
// is first written after MMA (1) completes
constexpr unsigned oU = oS;
static_assert(2 * kCtElems * 27 * 16 <= 128 * kSld * 4, "nodal staging must fit in the TMEM staging");
constexpr unsigned oLt = oS + 128 * kSld * 4;               // int[16][27]
constexpr unsigned oX = oLt + kCtElems * 27 * 4;            // float[16][24] corner coordinates
constexpr unsigned oDsp = oX + kCtElems * 24 * 4;           // float[3][8][8]
constexpr unsigned oW = oDsp + 3 * 8 * 8 * 4;               // float[8]
constexpr unsigned oBar = (oW + 8 * 4 + 15) & ~15u;         // 2 mbarriers
constexpr unsigned oSlot = oBar + 16;                       // TMEM base address
constexpr unsigned kCtSmem = oSlot + 16;

// Byte offset of (row r, k) inside one K-step tile of R rows, k in 0..7.
__device__ __forceinline__ unsigned kmaj(int R, int r, int k) {
  return (unsigned)((((k >> 2) * R + r) << 4) + ((k & 3) << 2));
}
__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xffffe000u); }
__device__ __forceinline__ void put_split(unsigned char* hi, unsigned char* lo, unsigned off, float x) {
  const float h = tf32_hi(x);
  *reinterpret_cast<float*>(hi + off) = h;
  *reinterpret_cast<float*>(lo + off) = x - h;
}

// TF32 x TF32 -> FP32, both operands K-major, M = 128, N = 32.
constexpr unsigned kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_tf32(unsigned tmem_d, unsigned long long a, unsigned long long b,
                                          unsigned accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdescTf32), "r"(accumulate));
}

// *p += (x, y, z, w) as one 16-byte vector reduction in L2
__device__ __forceinline__ void red_add_v4(float4* p, float x, float y, float z, float w) {
  asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(x), "f"(y), "f"(z),
               "f"(w)
               : "memory");
}

__global__ void __launch_bounds__(kCtThreads) k_convect_tc(ConvArgs<float> a, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *A1h = smem + oA1h, *A1l = smem + oA1l, *B1h = smem + oB1h, *B1l = smem + oB1l;
  unsigned char *A2h = smem + oA2h, *A2l = smem + oA2l, *B2h = smem + oB2h, *B2l = smem + oB2l;
  float(*S)[kSld] = reinterpret_cast<float(*)[kSld]>(smem + oS);
  float4(*sU)[27] = reinterpret_cast<float4(*)[27]>(smem + oU);
  float4(*sP)[27] = sU + kCtElems;
  int(*lt)[27] = reinterpret_cast<int(*)[27]>(smem + oLt);
  float(*X)[24] = reinterpret_cast<float(*)[24]>(smem + oX);
  float(*sdSp)[8][8] = reinterpret_cast<float(*)[8][8]>(smem + oDsp);
  float* sw = reinterpret_cast<float*>(smem + oW);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + oBar);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(smem + oSlot);
  const int t = threadIdx.x, warp = t >> 5;

  // operand tiles start at zero (padding rows and K columns stay zero); the
  // constant basis tiles, split into hi and lo
  for (unsigned i = t; i < oS / 16; i += kCtThreads) reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  const Basis* B = a.basis;
  for (int i = t; i < 32 * 32; i += kCtThreads) {
    const int n = i >> 5, j = i & 31, s = n >> 3, k = n & 7;  // column (s, k) of (1), node j
    const double v = j < 27 ? (s == 0 ? B->Sv[k][j] : B->dSv[s - 1][k][j]) : 0.0;
    put_split(B1h, B1l, (unsigned)(j >> 3) * 1024u + kmaj(32, n, j & 7), (float)v);
  }
  for (int i = t; i < 32 * 8; i += kCtThreads) {
    const int n = i >> 3, k = i & 7;  // node n, Gauss point k of (2)
    put_split(B2h, B2l, kmaj(32, n, k), n < 27 ? (float)B->Sv[k][n] : 0.f);
  }
  for (int i = t; i < 3 * 8 * 8; i += kCtThreads) sdSp[i / 64][(i / 8) % 8][i % 8] = (float)B->dSp[i / 64][(i / 8) % 8][i % 8];
  if (t < 8) sw[t] = (float)B->w[t];
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(tmem_slot, kCtCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  const unsigned trow = tmem + ((unsigned)(32 * warp) << 16);  // this warp's TMEM lanes

  const int r = t;                   // the row of (1) and (2) this thread reads back
  const int re = r >> 3, rq = r & 7;  // its element slot and quantity / Gauss point / component
  const int ntiles = (a.e_end - a.e_begin + kCtElems - 1) / kCtElems;
  bool ok = true;
  int it = 0, pending = 0;  // the barrier whose wait gave up
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, it++) {
    const int p0 = a.e_begin + tile * kCtElems;
    const int cnt = min(kCtElems, a.e_end - p0);
    // connectivity (contiguous rows), then nodal values and corner
    // coordinates with consecutive threads on consecutive elements
    for (int i = t; i < kCtElems * 27; i += kCtThreads) {
      const int e = i / 27, j = i % 27;
      lt[e][j] = e < cnt ? __ldg(a.ltog + (size_t)(p0 + e) * 27 + j) : 0;
    }
    __syncthreads();
    for (int i = t; i < kCtElems * 27; i += kCtThreads) {
      const int e = i % kCtElems, j = i / kCtElems;
      if (e < cnt) {
        const int node = lt[e][j];
        sU[e][j] = __ldg(a.un + node);
        sP[e][j] = __ldg(a.uprev + node);
      } else {
        sU[e][j] = make_float4(0.f, 0.f, 0.f, 0.f);
        sP[e][j] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    for (int i = t; i < kCtElems * 24; i += kCtThreads) {
      const int e = i % kCtElems, c = i / kCtElems;
      X[e][c] = e < cnt ? (float)__ldg(a.coord + 3 * (size_t)lt[e][c / 3] + c % 3) : 0.f;
    }
    __syncthreads();
    // operand A of (1): 16-byte row segments (element e, quantity q, K-step
    // s, half h), consecutive threads on consecutive rows
    for (int i = t; i < kCtElems * 6 * 8; i += kCtThreads) {
      const int q = i % 6, e = (i / 6) % kCtElems, sh = i / (6 * kCtElems), s = sh >> 1, h = sh & 1;
      const int j0 = 8 * s + 4 * h;
      float v[4];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int j = j0 + c;
        float x = 0.f;
        if (j < 27) {
          const float4 u = q < 3 ? sU[e][j] : sP[e][j];
          const int qq = q < 3 ? q : q - 3;
          x = qq == 0 ? u.x : (qq == 1 ? u.y : u.z);
        }
        v[c] = x;
      }
      float4 hv, lv;
      hv.x = tf32_hi(v[0]), hv.y = tf32_hi(v[1]), hv.z = tf32_hi(v[2]), hv.w = tf32_hi(v[3]);
      lv.x = v[0] - hv.x, lv.y = v[1] - hv.y, lv.z = v[2] - hv.z, lv.w = v[3] - hv.w;
      const unsigned off = (unsigned)s * 4096u + kmaj(128, 8 * e + q, 4 * h);
      *reinterpret_cast<float4*>(A1h + off) = hv;
      *reinterpret_cast<float4*>(A1l + off) = lv;
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const unsigned long long ah = umma_desc(smem_u32(A1h + s * 4096), 2048u, 128u);
        const unsigned long long al = umma_desc(smem_u32(A1l + s * 4096), 2048u, 128u);
        const unsigned long long bh = umma_desc(smem_u32(B1h + s * 1024), 512u, 128u);
        const unsigned long long bl = umma_desc(smem_u32(B1l + s * 1024), 512u, 128u);
        umma_tf32(tmem, ah, bh, s > 0 ? 1u : 0u);
        umma_tf32(tmem, ah, bl, 1u);
        umma_tf32(tmem, al, bh, 1u);
      }
      umma_commit(&bar[0]);
    }
    __syncwarp();
    ok = __syncthreads_and(mbar_wait_bounded(&bar[0], (unsigned)(it & 1), kCtWaitNs));
    tc_fence_after();
    if (!ok) {
      pending = 0;
      break;
    }
    {
      float v[16];
      tmem_ld16(trow, v);
#pragma unroll
      for (int c = 0; c < 16; c++) S[r][c] = v[c];
      tmem_ld16(trow + 16, v);
#pragma unroll
      for (int c = 0; c < 16; c++) S[r][16 + c] = v[c];
    }
    __syncwarp();  // an element's 8 rows belong to one warp
    {
      // Gauss point k = rq of element slot re: the convective products
      const int e = re, k = rq;
      float ck[3] = {0.f, 0.f, 0.f};
      if (e < cnt) {
        const float u0[3] = {S[8 * e][k], S[8 * e + 1][k], S[8 * e + 2][k]};
        float gr[3][3];  // gr[a][d] = d uprev^d / d xi_a
#pragma unroll
        for (int aa = 0; aa < 3; aa++)
#pragma unroll
          for (int d = 0; d < 3; d++) gr[aa][d] = S[8 * e + 3 + d][8 * (1 + aa) + k];
        float J[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int jj = 0; jj < 3; jj++) {
            float s = 0.f;
#pragma unroll
            for (int m = 0; m < 8; m++) s += sdSp[i][k][m] * X[e][3 * m + jj];
            J[i][jj] = s;
          }
        const float det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) +
                          J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
                          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        const float inv = 1.f / det;
        float iJ[3][3];
        iJ[0][0] = (J[1][1] * J[2][2] - J[2][1] * J[1][2]) * inv;
        iJ[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) * inv;
        iJ[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * inv;
        iJ[1][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]) * inv;
        iJ[1][1] = (J[2][2] * J[0][0] - J[2][0] * J[0][2]) * inv;
        iJ[1][2] = -(J[1][2] * J[0][0] - J[1][0] * J[0][2]) * inv;
        iJ[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * inv;
        iJ[2][1] = -(J[2][1] * J[0][0] - J[2][0] * J[0][1]) * inv;
        iJ[2][2] = (J[1][1] * J[0][0] - J[1][0] * J[0][1]) * inv;
        const float f = det * sw[k];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const float gx = iJ[0][0] * gr[0][d] + iJ[0][1] * gr[1][d] + iJ[0][2] * gr[2][d];
          const float gy = iJ[1][0] * gr[0][d] + iJ[1][1] * gr[1][d] + iJ[1][2] * gr[2][d];
          const float gz = iJ[2][0] * gr[0][d] + iJ[2][1] * gr[1][d] + iJ[2][2] * gr[2][d];
          ck[d] = (u0[0] * gx + u0[1] * gy + u0[2] * gz) * f;
        }
      }
      // operand A of (2): rows (e, d), K = Gauss point k
#pragma unroll
      for (int d = 0; d < 3; d++) put_split(A2h, A2l, kmaj(128, 8 * e + d, k), ck[d]);
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      const unsigned long long ah = umma_desc(smem_u32(A2h), 2048u, 128u);
      const unsigned long long al = umma_desc(smem_u32(A2l), 2048u, 128u);
      const unsigned long long bh = umma_desc(smem_u32(B2h), 512u, 128u);
      const unsigned long long bl = umma_desc(smem_u32(B2l), 512u, 128u);
      umma_tf32(tmem + 32, ah, bh, 0u);
      umma_tf32(tmem + 32, ah, bl, 1u);
      umma_tf32(tmem + 32, al, bh, 1u);
      umma_commit(&bar[1]);
    }
    __syncwarp();
    ok = __syncthreads_and(mbar_wait_bounded(&bar[1], (unsigned)(it & 1), kCtWaitNs));
    tc_fence_after();
    if (!ok) {
      pending = 1;
      break;
    }
    {
      // row (e, d): R1e_i^d over the nodes i
      float v[16];
      tmem_ld16(trow + 32, v);
#pragma unroll
      for (int c = 0; c < 16; c++) S[r][c] = v[c];
      tmem_ld16(trow + 48, v);
#pragma unroll
      for (int c = 0; c < 16; c++) S[r][16 + c] = v[c];
    }
    __syncwarp();
    if (re < cnt) {
      // nodes i = rq, rq + 8, ... of element slot re, all three components
      for (int i = rq; i < 27; i += 8)
        red_add_v4(a.r1f + lt[re][i], -S[8 * re][i], -S[8 * re + 1][i], -S[8 * re + 2][i], 0.f);
    }
    tc_fence_before();
    __syncthreads();
  }
  if (!ok) {
    // a bounded wait gave up: report it, give the MMAs still in flight one
    // more bounded wait, then release the accumulator columns
    if (t == 0) {
      atomicExch(err, 1);
      mbar_wait_bounded(&bar[pending], (unsigned)(it & 1), kCtWaitNs);
    }
    tc_fence_before();
    __syncthreads();
  }
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, kCtCols);
}

}  // namespace

bool convect_tc_supported(const ConvArgs<float>& a) {
  return a.ngp == 8 && a.r1f && !a.plain && !a.elist && a.e_end > a.e_begin;
}

cudaError_t launch_convect_tc(const ConvArgs<float>& a, int* err, int num_sms, cudaStream_t s) {
  if (!convect_tc_supported(a) || !err) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_convect_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCtSmem);
  // all of the unified L1 as shared memory: three 72 KB blocks per SM
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_convect_tc, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  // blocks per SM from the shared memory (the occupancy query answered one
  // block per SM for this kernel, where three fit)
  int dev = 0, smem_sm = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (e != cudaSuccess) return e;
  int per_sm = smem_sm / (int)(kCtSmem + 1024);  // 1 KB reserved per block
  per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
  const int ntiles = (a.e_end - a.e_begin + kCtElems - 1) / kCtElems;
  int grid = num_sms * per_sm;
  if (grid > ntiles) grid = ntiles;
  k_convect_tc<<<grid, kCtThreads, kCtSmem, s>>>(a, err);
  return cudaGetLastError();
}

}  // namespace cfd
