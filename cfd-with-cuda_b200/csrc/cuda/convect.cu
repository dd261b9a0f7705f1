// Convection right-hand side R1 = -A(Un) UnpHalf_prev, matrix-free
// (calculateMatrixA, blascoCodinaHuerta.cpp:3520-3685; calcAndAssembleMatrixA,
// CUDAcodes.cu:695-899).
//
// The reference forms the 27x27 element matrix
//   Ae[i][j] = sum_k (u0_k . grad Sv_j(k)) Sv_i(k) detJ_k w_k
// and multiplies it with the element's UnpHalf_prev values.  The same sum is
// evaluated here in factored form, which needs no Ae:
//   c_k^d  = u0_k . grad(uprev^d)(k)       (u0_k interpolated from Un)
//   R1e_i^d = sum_k Sv_i(k) detJ_k w_k c_k^d
// with grad(uprev^d)(k) = J_k^{-1} (sum_j dSv_j(k) uprev_j^d), J_k rebuilt
// from the 8 corner coordinates.  Work per element is about 30x fewer flops
// than the Ae form, so the kernel is bound by the L1 data pipe: the gathers
// of Un / UnpHalf_prev and the shared-memory operand reads of the
// Gauss-point sums.  The layout keeps both low:
// - a block takes EPB consecutive elements; their connectivity is read
//   element by element (27 contiguous ints), then the nodal values and
//   corner coordinates are gathered with consecutive threads on consecutive
//   elements at the same local node, which for a structured numbering are
//   neighbouring nodes (few cache lines per warp request);
// - TPE threads share an element, each owning GPT Gauss points: a nodal
//   value read from shared memory serves GPT Gauss points, and a warp reads
//   the basis values of only TPE Gauss points per node at a time;
// - the scatter again runs consecutive threads over consecutive elements.
// Results are scattered with FP64 atomics (no element colouring; in mixed
// precision as one FP32 16-byte vector reduction per element node into an
// FP32 copy of the term), or, in deterministic mode, one colour per launch
// with plain adds.  Every sum runs in the same order whatever the layout:
// over nodes j for a Gauss point, over Gauss points k for a node.
#include "kernels.h"

namespace cfd {

namespace {

constexpr int kConvThreads = 128;

// *p += (x, y, z, w) as one 16-byte vector reduction in L2 (sm_90 and newer)
__device__ __forceinline__ void red_add_v4_f32(float4* p, float x, float y, float z, float w) {
  asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(x), "f"(y), "f"(z),
               "f"(w)
               : "memory");
}

// Four values of T read from shared memory by one vector load.
template <class T>
struct alignas(4 * sizeof(T)) Quad {
  T x, y, z, w;
};

// Shared-memory carve-up of one block (byte offsets, each a multiple of 32,
// the alignment of Quad<double>).
constexpr size_t round32(size_t b) { return (b + 31) & ~size_t(31); }
template <class T, int TPE, int GPT>
struct ConvSmem {
  static constexpr int EPB = kConvThreads / TPE;
  static constexpr int NG = TPE * GPT;  // Gauss points a block can hold
  static constexpr int NGP = NG + 1;    // padded row of cc (no bank conflicts across elements)
  static constexpr size_t sB = 0;                                                // Quad<T>[NG][27]
  static constexpr size_t sdSp = sB + round32(sizeof(Quad<T>) * NG * 27);       // T[3][NG][8]
  static constexpr size_t sw = sdSp + round32(sizeof(T) * 3 * NG * 8);           // T[NG]
  static constexpr size_t u0 = sw + round32(sizeof(T) * NG);                     // Quad<T>[EPB][27]
  static constexpr size_t up = u0 + round32(sizeof(Quad<T>) * EPB * 27);         // Quad<T>[EPB][27]
  static constexpr size_t cc = up + round32(sizeof(Quad<T>) * EPB * 27);         // Quad<T>[EPB][NGP]
  static constexpr size_t X = cc + round32(sizeof(Quad<T>) * EPB * NGP);         // T[EPB][25]
  static constexpr size_t lt = X + round32(sizeof(T) * EPB * 25);                // int[EPB][27]
  static constexpr size_t bytes = lt + round32(sizeof(int) * EPB * 27);
};

template <class T, int TPE, int GPT>
__global__ void __launch_bounds__(kConvThreads) k_convect(ConvArgs<T> a) {
  using L = ConvSmem<T, TPE, GPT>;
  constexpr int EPB = L::EPB, NG = L::NG, NGP = L::NGP;
  extern __shared__ __align__(32) unsigned char smem[];
  auto sB = reinterpret_cast<Quad<T>(*)[27]>(smem + L::sB);  // {Sv, dSv/dxi, dSv/deta, dSv/dzeta}
  auto sdSp = reinterpret_cast<T(*)[NG][8]>(smem + L::sdSp);
  T* sw = reinterpret_cast<T*>(smem + L::sw);
  auto u0 = reinterpret_cast<Quad<T>(*)[27]>(smem + L::u0);
  auto up = reinterpret_cast<Quad<T>(*)[27]>(smem + L::up);
  auto cc = reinterpret_cast<Quad<T>(*)[NGP]>(smem + L::cc);
  auto X = reinterpret_cast<T(*)[25]>(smem + L::X);  // corner m, coordinate d at 3 m + d
  auto lt = reinterpret_cast<int(*)[27]>(smem + L::lt);
  const int t = threadIdx.x, ngp = a.ngp;
  const Basis* B = a.basis;
  for (int i = t; i < NG * 27; i += blockDim.x) {
    const int k = i / 27, j = i % 27;
    sB[k][j] = k < ngp ? Quad<T>{(T)B->Sv[k][j], (T)B->dSv[0][k][j], (T)B->dSv[1][k][j], (T)B->dSv[2][k][j]}
                       : Quad<T>{T(0), T(0), T(0), T(0)};
  }
  for (int i = t; i < NG * 8; i += blockDim.x) {
    const int k = i / 8, m = i % 8;
    for (int d = 0; d < 3; d++) sdSp[d][k][m] = k < ngp ? (T)B->dSp[d][k][m] : T(0);
  }
  for (int i = t; i < NG; i += blockDim.x) sw[i] = i < ngp ? (T)B->w[i] : T(0);
  const int el = t / TPE, tk = t % TPE;
  // element of local slot l in this pass (-1 past the range)
  auto elem_of = [&](int p0, int l) -> int {
    const int pos = p0 + l;
    return pos < a.e_end ? (a.elist ? __ldg(a.elist + pos) : pos) : -1;
  };
  for (int p0 = a.e_begin + blockIdx.x * EPB; p0 < a.e_end; p0 += gridDim.x * EPB) {
    __syncthreads();
    // connectivity, element by element (contiguous rows of ltog)
    for (int idx = t; idx < EPB * 27; idx += blockDim.x) {
      const int l = idx / 27, i = idx % 27, e = elem_of(p0, l);
      lt[l][i] = e >= 0 ? __ldg(a.ltog + (size_t)e * 27 + i) : 0;
    }
    __syncthreads();
    // nodal values and corner coordinates, consecutive threads on
    // consecutive elements at one local node
    for (int idx = t; idx < EPB * 27; idx += blockDim.x) {
      const int l = idx % EPB, i = idx / EPB;
      if (elem_of(p0, l) >= 0) {
        const int node = lt[l][i];
        const auto u = ldgv(a.un + node);
        const auto p = ldgv(a.uprev + node);
        u0[l][i] = Quad<T>{(T)u.x, (T)u.y, (T)u.z, T(0)};
        up[l][i] = Quad<T>{(T)p.x, (T)p.y, (T)p.z, T(0)};
      }
    }
    for (int idx = t; idx < EPB * 24; idx += blockDim.x) {
      const int l = idx % EPB, r = idx / EPB;
      if (elem_of(p0, l) >= 0) X[l][r] = (T)__ldg(a.coord + 3 * (size_t)lt[l][r / 3] + r % 3);
    }
    __syncthreads();
    const int e = elem_of(p0, el);
    if (e >= 0) {
      // u0 at the thread's Gauss points k = tk + TPE g and reference-space
      // gradients of uprev (g[.][a][d] = d uprev^d / d xi_a), summed over j
      T uk[GPT][3], gr[GPT][3][3];
#pragma unroll
      for (int g = 0; g < GPT; g++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          uk[g][d] = 0;
          gr[g][0][d] = gr[g][1][d] = gr[g][2][d] = 0;
        }
#pragma unroll 3
      for (int j = 0; j < 27; j++) {
        const Quad<T> ua = u0[el][j], ub = up[el][j];
#pragma unroll
        for (int g = 0; g < GPT; g++) {
          const Quad<T> bs = sB[tk + TPE * g][j];
          uk[g][0] += bs.x * ua.x; uk[g][1] += bs.x * ua.y; uk[g][2] += bs.x * ua.z;
          gr[g][0][0] += bs.y * ub.x; gr[g][0][1] += bs.y * ub.y; gr[g][0][2] += bs.y * ub.z;
          gr[g][1][0] += bs.z * ub.x; gr[g][1][1] += bs.z * ub.y; gr[g][1][2] += bs.z * ub.z;
          gr[g][2][0] += bs.w * ub.x; gr[g][2][1] += bs.w * ub.y; gr[g][2][2] += bs.w * ub.z;
        }
      }
#pragma unroll
      for (int g = 0; g < GPT; g++) {
        const int k = tk + TPE * g;
        if (k >= ngp) {
          cc[el][k] = Quad<T>{T(0), T(0), T(0), T(0)};
          continue;
        }
        // Jacobian of the trilinear corner map at Gauss point k
        T J[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int jj = 0; jj < 3; jj++) {
            T s = 0;
#pragma unroll
            for (int m = 0; m < 8; m++) s += sdSp[i][k][m] * X[el][3 * m + jj];
            J[i][jj] = s;
          }
        const T det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) +
                      J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
                      J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        const T inv = T(1) / det;
        T iJ[3][3];
        iJ[0][0] = (J[1][1] * J[2][2] - J[2][1] * J[1][2]) * inv;
        iJ[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) * inv;
        iJ[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * inv;
        iJ[1][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]) * inv;
        iJ[1][1] = (J[2][2] * J[0][0] - J[2][0] * J[0][2]) * inv;
        iJ[1][2] = -(J[1][2] * J[0][0] - J[1][0] * J[0][2]) * inv;
        iJ[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * inv;
        iJ[2][1] = -(J[2][1] * J[0][0] - J[2][0] * J[0][1]) * inv;
        iJ[2][2] = (J[1][1] * J[0][0] - J[1][0] * J[0][1]) * inv;
        const T f = det * sw[k];
        T ck[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          // physical gradient of uprev^d: grad_i = sum_a iJ[i][a] g[a][d]
          const T gx = iJ[0][0] * gr[g][0][d] + iJ[0][1] * gr[g][1][d] + iJ[0][2] * gr[g][2][d];
          const T gy = iJ[1][0] * gr[g][0][d] + iJ[1][1] * gr[g][1][d] + iJ[1][2] * gr[g][2][d];
          const T gz = iJ[2][0] * gr[g][0][d] + iJ[2][1] * gr[g][1][d] + iJ[2][2] * gr[g][2][d];
          ck[d] = (uk[g][0] * gx + uk[g][1] * gy + uk[g][2] * gz) * f;
        }
        cc[el][k] = Quad<T>{ck[0], ck[1], ck[2], T(0)};
      }
    }
    __syncthreads();
    // R1e_i^d = sum_k Sv_i(k) c_k^d, consecutive threads on consecutive
    // elements at one local node
    for (int idx = t; idx < EPB * 27; idx += blockDim.x) {
      const int l = idx % EPB, i = idx / EPB;
      if (elem_of(p0, l) < 0) continue;
      T s0 = 0, s1 = 0, s2 = 0;
      for (int k = 0; k < ngp; k++) {
        const T sv = sB[k][i].x;
        const Quad<T> ck = cc[l][k];
        s0 += sv * ck.x;
        s1 += sv * ck.y;
        s2 += sv * ck.z;
      }
      const int node = lt[l][i];
      if constexpr (sizeof(T) == 4) {
        if (a.r1f) {
          float4* df = a.r1f + node;
          if (a.plain) {
            float4 o = *df;
            o.x -= (float)s0;
            o.y -= (float)s1;
            o.z -= (float)s2;
            *df = o;
          } else {
            red_add_v4_f32(df, -(float)s0, -(float)s1, -(float)s2, 0.f);
          }
          continue;
        }
      }
      double4* dst = a.r1 + node;
      if (a.plain) {  // one colour per launch: no other element of it touches this node
        dst->x -= (double)s0;
        dst->y -= (double)s1;
        dst->z -= (double)s2;
      } else {
        atomicAdd(&dst->x, -(double)s0);
        atomicAdd(&dst->y, -(double)s1);
        atomicAdd(&dst->z, -(double)s2);
      }
    }
  }
}

template <class T, int TPE, int GPT>
cudaError_t launch_convect_cfg(const ConvArgs<T>& a, int ne, int num_sms, cudaStream_t s) {
  using L = ConvSmem<T, TPE, GPT>;
  auto k = k_convect<T, TPE, GPT>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kConvThreads, L::bytes);
  if (e != cudaSuccess) return e;
  int grid = (ne + L::EPB - 1) / L::EPB;
  const int cap = num_sms * (per_sm > 0 ? per_sm : 1);
  if (grid > cap) grid = cap;
  k<<<grid, kConvThreads, L::bytes, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

template <class T>
cudaError_t launch_convect(const ConvArgs<T>& a, int num_sms, cudaStream_t s) {
  const int ne = a.e_end - a.e_begin;
  if (ne <= 0) return cudaSuccess;
  if (a.ngp > kMaxNGP || a.ngp < 1) return cudaErrorInvalidValue;
  // 4 threads per element, 32 elements per block: 2 Gauss points per thread
  // at NGP 8, 7 at NGP 27
  if (a.ngp <= 8) return launch_convect_cfg<T, 4, 2>(a, ne, num_sms, s);
  return launch_convect_cfg<T, 4, 7>(a, ne, num_sms, s);
}

template cudaError_t launch_convect<double>(const ConvArgs<double>&, int, cudaStream_t);
template cudaError_t launch_convect<float>(const ConvArgs<float>&, int, cudaStream_t);

}  // namespace cfd
