// Fractional-step stage kernels (step1GPUpart, step2GPU, step3GPU,
// calculate_KtimesAcc_prevGPU and the convergence norms of CUDAcodes.cu:
// 946-1121).  Each stage is one pass over its SELL-32 operator(s) with the
// elementwise work fused into the epilogue, replacing the reference's 3-6
// library SpMVs plus 2-4 elementwise kernels and the temporary
// cudaMalloc/cudaFree of every call.
//
// One thread owns one row; a warp owns one 32-row slice, so the entry loop
// has a warp-uniform trip count, needs no shuffles, and every load of the
// matrix is a contiguous warp-wide segment.  Matrix values and columns are
// read with streaming (evict-first) loads so the gathered vectors stay in
// L2.  Matrix values are VT (double or float, accumulated in VT); vectors
// stay FP64.
#include "kernels.h"

namespace cfd {

namespace {

constexpr int kRowThreads = 256;

inline int rows_grid(long long rows) {
  long long g = (rows + kRowThreads - 1) / kRowThreads;
  return (int)(g < 1 ? 1 : g);
}

// step1: R1 = R1conv - K UnpHalf_prev - G Pn (blascoCodinaHuerta.cpp:
// 3745-3758), R1 = 0 at Dirichlet nodes (applyBC_Step1(2)),
// UnpHalf = Un + dt R1 MdInv (:3781-3783) -- the Dirichlet zeroing is the
// zero in minv_free.  Also writes d = UnpHalf/dt^2 - [iter>1] MdOrigInv KAcc,
// the input of step2 (blascoCodinaHuerta.cpp:3821-3832).
template <class VT>
__global__ void __launch_bounds__(kRowThreads) k_step1(Step1Args<VT> a) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= a.NN) return;
  const int s = row >> 5, l = row & 31;
  const double inv_dt2 = 1.0000000000000000 / (a.dt * a.dt);
  VT kx = 0, ky = 0, kz = 0, gx = 0, gy = 0, gz = 0;
  {
    const int b = __ldg(a.k_off + s), w = (__ldg(a.k_off + s + 1) - b) >> 5;
    const int* col = a.k_col + b + l;
    const VT* val = a.kval + b + l;
#pragma unroll 4
    for (int j = 0; j < w; j++) {
      const VT v = __ldcs(val + 32 * j);
      const auto x = ldgv(a.uprev + __ldcs(col + 32 * j));
      kx += v * (VT)x.x;
      ky += v * (VT)x.y;
      kz += v * (VT)x.z;
    }
  }
  {
    const int b = __ldg(a.g_off + s), w = (__ldg(a.g_off + s + 1) - b) >> 5;
    const int* col = a.g_col + b + l;
#pragma unroll 4
    for (int j = 0; j < w; j++) {
      const VT p = (VT)__ldg(a.pn + __ldcs(col + 32 * j));
      gx += __ldcs(a.g1 + b + l + 32 * j) * p;
      gy += __ldcs(a.g2 + b + l + 32 * j) * p;
      gz += __ldcs(a.g3 + b + l + 32 * j) * p;
    }
  }
  double4 rc;
  if (a.r1conv32) {
    const float4 f = a.r1conv32[row];
    rc = make_double4(f.x, f.y, f.z, 0.0);
  } else {
    rc = a.r1conv[row];
  }
  const double mf = a.minv_free[row];
  double rx = (rc.x - (double)kx) - (double)gx;
  double ry = (rc.y - (double)ky) - (double)gy;
  double rz = (rc.z - (double)kz) - (double)gz;
  if (mf == 0.0) rx = ry = rz = 0.0;  // Dirichlet node
  const double4 u = a.un[row];
  double4 h;
  h.x = u.x + a.dt * rx * mf;
  h.y = u.y + a.dt * ry * mf;
  h.z = u.z + a.dt * rz * mf;
  h.w = 0.0;
  a.unphalf[row] = h;
  if constexpr (sizeof(VT) == 4) a.unphalf_g[row] = to_f4(h);
  double4 d;
  d.x = inv_dt2 * h.x;
  d.y = inv_dt2 * h.y;
  d.z = inv_dt2 * h.z;
  d.w = 0.0;
  if (a.iter != 1) {
    const double mo = a.minv_orig[row];
    const double4 ka = a.kacc[row];
    d.x = d.x - mo * ka.x;
    d.y = d.y - mo * ka.y;
    d.z = d.z - mo * ka.z;
  }
  a.d[row] = d;
  if constexpr (sizeof(VT) == 4) a.d_g[row] = to_f4(d);
  if (a.r1out) a.r1out[row] = make_double4(rx, ry, rz, 0.0);
}

// out[p] = sum_d (G_d^T d_d)[p]; out[pin] = 0 when pin > 0
// (step2GPU's three transposed csrmv calls + applyPresBC, CUDAcodes.cu:1006-1011).
template <class VT>
__global__ void __launch_bounds__(kRowThreads) k_gt(GtArgs<VT> a) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= a.NNp) return;
  const int s = row >> 5, l = row & 31;
  const int b = __ldg(a.gt_off + s) + l, w = (__ldg(a.gt_off + s + 1) - __ldg(a.gt_off + s)) >> 5;
  VT acc = 0;
#pragma unroll 4
  for (int j = 0; j < w; j++) {
    const int e = b + 32 * j;
    const auto d = ldgv(a.d + __ldcs(a.gt_col + e));
    acc += __ldcs(a.gt1 + e) * (VT)d.x + __ldcs(a.gt2 + e) * (VT)d.y + __ldcs(a.gt3 + e) * (VT)d.z;
  }
  a.out[row] = (a.pin > 0 && row == a.pin) ? 0.0 : (double)acc;
}

// step3: R3 = -dt G Pdot - [iter>1] dt KAcc, R3 = 0 at Dirichlet nodes,
// Acc = R3 MdInv, Unp1 = UnpHalf + dt Acc (blascoCodinaHuerta.cpp:3920-3967)
// plus the partial sums of the convergence test (:2936-2961) and of the
// steady-state test (:3052-3057).
template <class VT>
__global__ void __launch_bounds__(kRowThreads) k_step3(Step3Args<VT> a) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const double inv_dt = 1.0000000000000000 / a.dt;
  double s_u2 = 0, s_du2 = 0, m_acc = 0;
  if (row < a.NN) {
    const int s = row >> 5, l = row & 31;
    const int b = __ldg(a.g_off + s) + l, w = (__ldg(a.g_off + s + 1) - __ldg(a.g_off + s)) >> 5;
    VT gx = 0, gy = 0, gz = 0;
#pragma unroll 4
    for (int j = 0; j < w; j++) {
      const int e = b + 32 * j;
      const VT p = (VT)__ldg(a.pdot + __ldcs(a.g_col + e));
      gx += __ldcs(a.g1 + e) * p;
      gy += __ldcs(a.g2 + e) * p;
      gz += __ldcs(a.g3 + e) * p;
    }
    double rx = -a.dt * (double)gx, ry = -a.dt * (double)gy, rz = -a.dt * (double)gz;
    if (a.iter != 1) {
      const double4 ka = a.kacc[row];
      rx = rx - a.dt * ka.x;
      ry = ry - a.dt * ka.y;
      rz = rz - a.dt * ka.z;
    }
    const double mf = a.minv_free[row];
    if (mf == 0.0) rx = ry = rz = 0.0;  // Dirichlet node
    const double4 acc = make_double4(rx * mf, ry * mf, rz * mf, 0.0);
    const double4 h = a.unphalf[row];
    const double4 u1 = make_double4(h.x + a.dt * acc.x, h.y + a.dt * acc.y, h.z + a.dt * acc.z, 0.0);
    a.acc[row] = acc;
    if constexpr (sizeof(VT) == 4) a.acc_g[row] = to_f4(acc);
    a.unp1[row] = u1;
    if (a.r3out) a.r3out[row] = make_double4(rx, ry, rz, 0.0);
    const double4 pv = a.unp1_prev[row];
    const double4 un = a.un[row];
    s_u2 = u1.x * u1.x + u1.y * u1.y + u1.z * u1.z;
    const double dx = u1.x - pv.x, dy = u1.y - pv.y, dz = u1.z - pv.z;
    s_du2 = dx * dx + dy * dy + dz * dz;
    m_acc = fmax(fabs((u1.x - un.x) * inv_dt), fmax(fabs((u1.y - un.y) * inv_dt), fabs((u1.z - un.z) * inv_dt)));
  }
  double v[2] = {s_u2, s_du2};
  m_acc = warp_max(m_acc);
  __shared__ double smax[32];
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = m_acc;
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    double m = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, smax[w]);
    a.part[blockIdx.x] = v[0];
    a.part[a.nblocks + blockIdx.x] = v[1];
    a.part[2 * a.nblocks + blockIdx.x] = m;
  }
}

template <class VT>
__global__ void __launch_bounds__(kRowThreads) k_spmv_k3(SpmvK3Args<VT> a) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= a.NN) return;
  const int s = row >> 5, l = row & 31;
  const int b = __ldg(a.off + s) + l, w = (__ldg(a.off + s + 1) - __ldg(a.off + s)) >> 5;
  VT sx = 0, sy = 0, sz = 0;
#pragma unroll 4
  for (int j = 0; j < w; j++) {
    const int e = b + 32 * j;
    const VT v = __ldcs(a.val + e);
    const auto x = ldgv(a.x + __ldcs(a.col + e));
    sx += v * (VT)x.x;
    sy += v * (VT)x.y;
    sz += v * (VT)x.z;
  }
  a.y[row] = make_double4((double)sx, (double)sy, (double)sz, 0.0);
}

__global__ void __launch_bounds__(kRowThreads) k_pressure_update(int n, double dt, const double* __restrict__ pn,
                                                                 const double* __restrict__ pdot,
                                                                 const double* __restrict__ pprev, double* pnp1,
                                                                 double* part, int nblocks) {
  double v[2] = {0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double p = pn[i] + dt * pdot[i];
    pnp1[i] = p;
    v[0] += p * p;
    double d = p - pprev[i];
    v[1] += d * d;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = v[0];
    part[nblocks + blockIdx.x] = v[1];
  }
}

// Fixed-order reduction of the per-block partials (deterministic).
__global__ void k_reduce_norms(const double* __restrict__ up, int nub, const double* __restrict__ pp, int npb,
                               double* out) {
  double v[4] = {0, 0, 0, 0};
  double m = 0;
  for (int i = threadIdx.x; i < nub; i += blockDim.x) {
    v[0] += up[i];
    v[1] += up[nub + i];
    m = fmax(m, up[2 * nub + i]);
  }
  for (int i = threadIdx.x; i < npb; i += blockDim.x) {
    v[2] += pp[i];
    v[3] += pp[npb + i];
  }
  m = warp_max(m);
  __shared__ double smax[32];
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = m;
  block_sum<4>(v);
  if (threadIdx.x == 0) {
    double mm = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) mm = fmax(mm, smax[w]);
    out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; out[3] = v[3]; out[4] = mm;
  }
}

template <class T>
__global__ void k_csr_to_sell(int nrows, const int* __restrict__ rp, const double* __restrict__ csr,
                              const int* __restrict__ off, T* sell) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const int nslices = (nrows + 31) >> 5;
  if (row >= nslices * 32) return;
  const int s = row >> 5, l = row & 31;
  const int b = off[s] + l, w = (off[s + 1] - off[s]) >> 5;
  const int cb = row < nrows ? rp[row] : 0, len = row < nrows ? rp[row + 1] - cb : 0;
  for (int j = 0; j < w; j++) sell[b + 32 * j] = j < len ? (T)csr[cb + j] : (T)0;
}

// SELL-32 pattern of a CSR pattern: slice widths (longest row of each
// 32-row slice), then the columns slice-column-major, a row shorter than its
// slice padded with its last column (0 for an empty row or a row past the
// end).
__global__ void k_sell_widths(int nrows, const int* __restrict__ rp, int* __restrict__ width) {
  const int ns = (nrows + 31) >> 5;
  for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < ns; sl += gridDim.x * blockDim.x) {
    int w = 0;
    for (int r = 32 * sl; r < min(nrows, 32 * sl + 32); r++) w = max(w, rp[r + 1] - rp[r]);
    width[sl] = w;
  }
}
__global__ void k_sell_cols(int nrows, const int* __restrict__ rp, const int* __restrict__ col,
                            const int* __restrict__ off, int* __restrict__ scol) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const int nslices = (nrows + 31) >> 5;
  if (row >= nslices * 32) return;
  const int sl = row >> 5, l = row & 31;
  const int b = off[sl] + l, w = (off[sl + 1] - off[sl]) >> 5;
  const int cb = row < nrows ? rp[row] : 0, len = row < nrows ? rp[row + 1] - cb : 0;
  const int padc = len > 0 ? col[cb + len - 1] : 0;
  for (int j = 0; j < w; j++) scol[b + 32 * j] = j < len ? col[cb + j] : padc;
}

__global__ void k_blocks_to_vec4(int NN, const double* __restrict__ b, double4* v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += gridDim.x * blockDim.x)
    v[i] = make_double4(b[i], b[(size_t)NN + i], b[2 * (size_t)NN + i], 0.0);
}
__global__ void k_vec4_to_blocks(int NN, const double4* __restrict__ v, double* b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += gridDim.x * blockDim.x) {
    double4 x = v[i];
    b[i] = x.x;
    b[(size_t)NN + i] = x.y;
    b[2 * (size_t)NN + i] = x.z;
  }
}
__global__ void k_apply_bc(int n, const int* __restrict__ nodes, const double* __restrict__ uvw, double4* u) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    u[nodes[i]] = make_double4(uvw[3 * (size_t)i], uvw[3 * (size_t)i + 1], uvw[3 * (size_t)i + 2], 0.0);
}

inline int ew_grid(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

template <class VT>
cudaError_t launch_step1(const Step1Args<VT>& a, int, cudaStream_t s) {
  k_step1<VT><<<rows_grid(a.NN), kRowThreads, 0, s>>>(a);
  return cudaGetLastError();
}
template <class VT>
cudaError_t launch_gt(const GtArgs<VT>& a, int, cudaStream_t s) {
  k_gt<VT><<<rows_grid(a.NNp), kRowThreads, 0, s>>>(a);
  return cudaGetLastError();
}
int step3_blocks(int NN, int) { return rows_grid(NN); }
template <class VT>
cudaError_t launch_step3(const Step3Args<VT>& a, cudaStream_t s) {
  k_step3<VT><<<a.nblocks, kRowThreads, 0, s>>>(a);
  return cudaGetLastError();
}
template <class VT>
cudaError_t launch_spmv_k3(const SpmvK3Args<VT>& a, int, cudaStream_t s) {
  k_spmv_k3<VT><<<rows_grid(a.NN), kRowThreads, 0, s>>>(a);
  return cudaGetLastError();
}
int pupdate_blocks(int NNp, int num_sms) { return ew_grid(NNp) < num_sms * 4 ? ew_grid(NNp) : num_sms * 4; }
cudaError_t launch_pressure_update(int NNp, double dt, const double* pn, const double* pdot, const double* pprev,
                                   double* pnp1, double* part, int nblocks, cudaStream_t s) {
  k_pressure_update<<<nblocks, kRowThreads, 0, s>>>(NNp, dt, pn, pdot, pprev, pnp1, part, nblocks);
  return cudaGetLastError();
}
cudaError_t launch_reduce_norms(const double* upart, int nub, const double* ppart, int npb, double* out,
                                cudaStream_t s) {
  k_reduce_norms<<<1, 1024, 0, s>>>(upart, nub, ppart, npb, out);
  return cudaGetLastError();
}
cudaError_t launch_sell_widths(int nrows, const int* rp, int* width, cudaStream_t s) {
  const int ns = (nrows + 31) / 32;
  k_sell_widths<<<rows_grid(ns) < 4096 ? rows_grid(ns) : 4096, kRowThreads, 0, s>>>(nrows, rp, width);
  return cudaGetLastError();
}
cudaError_t launch_sell_cols(int nrows, const int* rp, const int* col, const int* off, int* scol, cudaStream_t s) {
  const int nslices = (nrows + 31) / 32;
  k_sell_cols<<<rows_grid((long long)nslices * 32), kRowThreads, 0, s>>>(nrows, rp, col, off, scol);
  return cudaGetLastError();
}
template <class T>
cudaError_t launch_csr_to_sell(int nrows, const int* rp, const double* csr, const int* off, T* sell, cudaStream_t s) {
  const int nslices = (nrows + 31) / 32;
  k_csr_to_sell<T><<<rows_grid((long long)nslices * 32), kRowThreads, 0, s>>>(nrows, rp, csr, off, sell);
  return cudaGetLastError();
}
__global__ void k_vec4_to_f32(int NN, const double4* __restrict__ v, float4* a, float4* b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += gridDim.x * blockDim.x) {
    const float4 f = to_f4(v[i]);
    a[i] = f;
    b[i] = f;
  }
}

cudaError_t launch_vec4_to_f32(int NN, const double4* v, float4* a, float4* b, cudaStream_t s) {
  k_vec4_to_f32<<<rows_grid(NN), kRowThreads, 0, s>>>(NN, v, a, b);
  return cudaGetLastError();
}

cudaError_t launch_blocks_to_vec4(int NN, const double* blocks, double4* v, cudaStream_t s) {
  k_blocks_to_vec4<<<ew_grid(NN), 256, 0, s>>>(NN, blocks, v);
  return cudaGetLastError();
}
cudaError_t launch_vec4_to_blocks(int NN, const double4* v, double* blocks, cudaStream_t s) {
  k_vec4_to_blocks<<<ew_grid(NN), 256, 0, s>>>(NN, v, blocks);
  return cudaGetLastError();
}
cudaError_t launch_apply_bc(int n, const int* nodes, const double* uvw, double4* u, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_apply_bc<<<ew_grid(n), 256, 0, s>>>(n, nodes, uvw, u);
  return cudaGetLastError();
}

template cudaError_t launch_step1<double>(const Step1Args<double>&, int, cudaStream_t);
template cudaError_t launch_step1<float>(const Step1Args<float>&, int, cudaStream_t);
template cudaError_t launch_gt<double>(const GtArgs<double>&, int, cudaStream_t);
template cudaError_t launch_gt<float>(const GtArgs<float>&, int, cudaStream_t);
template cudaError_t launch_step3<double>(const Step3Args<double>&, cudaStream_t);
template cudaError_t launch_step3<float>(const Step3Args<float>&, cudaStream_t);
template cudaError_t launch_spmv_k3<double>(const SpmvK3Args<double>&, int, cudaStream_t);
template cudaError_t launch_spmv_k3<float>(const SpmvK3Args<float>&, int, cudaStream_t);
template cudaError_t launch_csr_to_sell<double>(int, const int*, const double*, const int*, double*, cudaStream_t);
template cudaError_t launch_csr_to_sell<float>(int, const int*, const double*, const int*, float*, cudaStream_t);

}  // namespace cfd
