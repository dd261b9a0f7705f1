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
// from the 8 corner coordinates.  One thread per (element, Gauss point);
// elements and their gathered nodal values sit in shared memory; results are
// scattered with FP64 atomics (no element colouring; in mixed precision as
// one FP32 16-byte vector reduction per element node into an FP32 copy of
// the term), or, in deterministic mode, one colour per launch with plain
// adds in a fixed order.  Work per element is
// about 30x fewer flops than the Ae form, so the kernel is bound by the
// gathers of Un / UnpHalf_prev and the atomic scatter, not by arithmetic.
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

template <class T, int TPE>
__global__ void __launch_bounds__(kConvThreads) k_convect(ConvArgs<T> a) {
  constexpr int EPB = kConvThreads / TPE;
  constexpr int NG = TPE < kMaxNGP ? TPE : kMaxNGP;
  // operands of the Gauss-point loops packed four to a vector load: the
  // loops are bound by shared-memory instructions, not by their FMAs
  __shared__ Quad<T> sB[NG][27];  // {Sv, dSv/dxi, dSv/deta, dSv/dzeta}
  __shared__ T sdSp[3][NG][8];
  __shared__ T sw[NG];
  __shared__ Quad<T> u0[EPB][27];
  __shared__ Quad<T> up[EPB][27];
  __shared__ T X[EPB][8][3];
  __shared__ Quad<T> cc[EPB][NG];
  __shared__ int lt[EPB][27];
  const int t = threadIdx.x, ngp = a.ngp;
  const Basis* B = a.basis;
  for (int i = t; i < ngp * 27; i += blockDim.x) {
    int k = i / 27, j = i % 27;
    sB[k][j] = Quad<T>{(T)B->Sv[k][j], (T)B->dSv[0][k][j], (T)B->dSv[1][k][j], (T)B->dSv[2][k][j]};
  }
  for (int i = t; i < ngp * 8; i += blockDim.x) {
    int k = i / 8, m = i % 8;
    sdSp[0][k][m] = (T)B->dSp[0][k][m];
    sdSp[1][k][m] = (T)B->dSp[1][k][m];
    sdSp[2][k][m] = (T)B->dSp[2][k][m];
  }
  for (int i = t; i < ngp; i += blockDim.x) sw[i] = (T)B->w[i];
  const int el = t / TPE, tk = t % TPE;
  // element of local slot l in this pass (-1 past the range)
  auto elem_of = [&](int p0, int l) -> int {
    const int pos = p0 + l;
    return pos < a.e_end ? (a.elist ? __ldg(a.elist + pos) : pos) : -1;
  };
  for (int p0 = a.e_begin + blockIdx.x * EPB; p0 < a.e_end; p0 += gridDim.x * EPB) {
    __syncthreads();
    for (int idx = t; idx < EPB * 27; idx += blockDim.x) {
      int l = idx / 27, i = idx % 27, e = elem_of(p0, l);
      if (e >= 0) {
        int node = __ldg(a.ltog + (size_t)e * 27 + i);
        lt[l][i] = node;
        const auto u = ldgv(a.un + node);
        const auto p = ldgv(a.uprev + node);
        u0[l][i] = Quad<T>{(T)u.x, (T)u.y, (T)u.z, T(0)};
        up[l][i] = Quad<T>{(T)p.x, (T)p.y, (T)p.z, T(0)};
      }
    }
    __syncthreads();
    for (int idx = t; idx < EPB * 24; idx += blockDim.x) {
      int l = idx / 24, r = idx % 24, e = elem_of(p0, l);
      if (e >= 0) X[l][r / 3][r % 3] = (T)__ldg(a.coord + 3 * (size_t)lt[l][r / 3] + r % 3);
    }
    __syncthreads();
    const int e = elem_of(p0, el);
    if (e >= 0 && tk < ngp) {
      const int k = tk;
      // Jacobian of the trilinear corner map at Gauss point k
      T J[3][3];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
          T s = 0;
#pragma unroll
          for (int m = 0; m < 8; m++) s += sdSp[i][k][m] * X[el][m][j];
          J[i][j] = s;
        }
      T det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) + J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
              J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
      T inv = T(1) / det;
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
      // u0 at the Gauss point and reference-space gradients of uprev
      T uk[3] = {0, 0, 0};
      T g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // g[a][d] = d uprev^d / d xi_a
#pragma unroll 3
      for (int j = 0; j < 27; j++) {
        const Quad<T> bs = sB[k][j], ua = u0[el][j], ub = up[el][j];
        const T sv = bs.x, d0 = bs.y, d1 = bs.z, d2 = bs.w;
        const T a0 = ua.x, a1 = ua.y, a2 = ua.z;
        const T b0 = ub.x, b1 = ub.y, b2 = ub.z;
        uk[0] += sv * a0; uk[1] += sv * a1; uk[2] += sv * a2;
        g[0][0] += d0 * b0; g[0][1] += d0 * b1; g[0][2] += d0 * b2;
        g[1][0] += d1 * b0; g[1][1] += d1 * b1; g[1][2] += d1 * b2;
        g[2][0] += d2 * b0; g[2][1] += d2 * b1; g[2][2] += d2 * b2;
      }
      const T f = det * sw[k];
      T ck[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        // physical gradient of uprev^d: grad_i = sum_a iJ[i][a] g[a][d]
        T gx = iJ[0][0] * g[0][d] + iJ[0][1] * g[1][d] + iJ[0][2] * g[2][d];
        T gy = iJ[1][0] * g[0][d] + iJ[1][1] * g[1][d] + iJ[1][2] * g[2][d];
        T gz = iJ[2][0] * g[0][d] + iJ[2][1] * g[1][d] + iJ[2][2] * g[2][d];
        ck[d] = (uk[0] * gx + uk[1] * gy + uk[2] * gz) * f;
      }
      cc[el][k] = Quad<T>{ck[0], ck[1], ck[2], T(0)};
    }
    __syncthreads();
    if (e >= 0) {
      for (int i = tk; i < 27; i += TPE) {
        T s0 = 0, s1 = 0, s2 = 0;
        for (int k = 0; k < ngp; k++) {
          const T sv = sB[k][i].x;
          const Quad<T> ck = cc[el][k];
          s0 += sv * ck.x;
          s1 += sv * ck.y;
          s2 += sv * ck.z;
        }
        if constexpr (sizeof(T) == 4) {
          if (a.r1f) {
            float4* df = a.r1f + lt[el][i];
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
        double4* dst = a.r1 + lt[el][i];
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
}

}  // namespace

template <class T>
cudaError_t launch_convect(const ConvArgs<T>& a, int num_sms, cudaStream_t s) {
  const int ne = a.e_end - a.e_begin;
  if (ne <= 0) return cudaSuccess;
  if (a.ngp <= 8) {
    constexpr int EPB = kConvThreads / 8;
    int grid = (ne + EPB - 1) / EPB;
    if (grid > num_sms * 12) grid = num_sms * 12;
    k_convect<T, 8><<<grid, kConvThreads, 0, s>>>(a);
  } else {
    constexpr int EPB = kConvThreads / 32;
    int grid = (ne + EPB - 1) / EPB;
    if (grid > num_sms * 12) grid = num_sms * 12;
    k_convect<T, 32><<<grid, kConvThreads, 0, s>>>(a);
  }
  return cudaGetLastError();
}

template cudaError_t launch_convect<double>(const ConvArgs<double>&, int, cudaStream_t);
template cudaError_t launch_convect<float>(const ConvArgs<float>&, int, cudaStream_t);

}  // namespace cfd
