// Host-visible launch interface of the solver kernels (plain pointers only).
//
// Device data layout (HBM):
//   velocity-sized vectors  double4 per node (x, y, z, pad = 0): one aligned
//                           32-byte sector per gathered node
//   pressure-sized vectors  double (or float for the FP32 inner solve)
//   K, G, G^T, Z            CSR (int32 rowptr/col, FP64 values) for assembly
//                           and download, plus a SELL-32 copy used by every
//                           per-step kernel: rows in slices of 32, each slice
//                           padded to its longest row and stored column-major
//                           (entry j of row r at off[r/32] + 32 j + r%32), so
//                           one thread owns one row and a warp-wide load of
//                           entry j is one contiguous 128/256-byte segment.
//                           Padding entries hold value 0 and a valid column.
//   gathered copies         CFD_MIXED keeps float4 copies (x, y, z, 0) of the
//                           velocity vectors that SpMVs and the convection
//                           gather (Un, UnpHalf_prev, Acc_prev, d): those
//                           kernels round every gathered value to FP32, so
//                           the copies give identical results at half the
//                           L1/L2 traffic of the 32-byte double4 gathers
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace cfd {

// Type of a gathered velocity vector: the float4 copy for FP32 operator
// values, the FP64 state itself otherwise.
template <class VT>
struct GatherVec {
  using type = double4;
};
template <>
struct GatherVec<float> {
  using type = float4;
};
template <class VT>
using GVec = typename GatherVec<VT>::type;

struct AsmArgs {
  int NE, ngp;
  const int* ltog;
  const double* coord;
  const Basis* basis;
  double viscosity, inv_density;
  const int *k_rp, *k_col;
  double* kval;
  const int *g_rp, *g_col;
  double *g1, *g2, *g3;
  double* msum;  // NN: row sums of M
  // element range [e_begin, e_end) of the list elist (null: ids themselves);
  // plain = 1: the range is one colour (no two elements share a node), so
  // the scatter adds without atomics and the sums are bitwise reproducible
  const int* elist;
  int e_begin, e_end, plain;
};
cudaError_t launch_assemble(const AsmArgs& a, int num_sms, cudaStream_t s);

// Gt values from G (Gt[k] = G[pos[k]]), MdOrigInv / MdInv-with-BC-mask.
cudaError_t launch_fill_gt(long long nnz, const int* pos, const double* g1, const double* g2,
                           const double* g3, double* gt1, double* gt2, double* gt3, cudaStream_t s);
cudaError_t launch_md_finalize(int NN, const double* msum, const unsigned char* bcmask, double* minv_orig,
                               double* minv_free, cudaStream_t s);

struct ZArgs {
  int NNp, maxrow, zeroP;
  const int *z_rp, *z_col;
  double* zval;
  double* zdiag;
  const int *gt_rp, *gt_col;
  const double *gt1, *gt2, *gt3;
  const int *g_rp, *g_col;
  const double *g1, *g2, *g3;
  const double* minv_orig;
};
cudaError_t launch_build_z(const ZArgs& a, cudaStream_t s);

cudaError_t launch_to_float(long long n, const double* in, float* out, cudaStream_t s);
cudaError_t launch_recip(long long n, const double* in, double* out64, float* out32, cudaStream_t s);

template <class T>
struct ConvArgs {
  int NE, ngp;
  const int* ltog;
  const double* coord;
  const Basis* basis;
  const GVec<T>* un;     // convecting velocity (time level n)
  const GVec<T>* uprev;  // UnpHalf_prev
  double4* r1;           // accumulates -A(un) uprev (zeroed by the caller)
  const int* elist;      // element range and plain scatter as in AsmArgs
  int e_begin, e_end, plain;
  // T = float only, may be null: accumulate into this FP32 copy instead of
  // r1 (zeroed by the caller; w stays 0), one 16-byte vector reduction per
  // element node instead of three FP64 atomics
  float4* r1f;
};
template <class T>
cudaError_t launch_convect(const ConvArgs<T>& a, int num_sms, cudaStream_t s);
// The same term with the per-element contractions on the tensor cores
// (tcgen05, TF32 split into hi + lo parts; convect_tc.cu): FP32 copies (r1f
// set), NGP = 8, no colouring.  *err (device, zeroed by the caller) is set
// when a bounded wait of the kernel gives up.
bool convect_tc_supported(const ConvArgs<float>& a);
cudaError_t launch_convect_tc(const ConvArgs<float>& a, int* err, int num_sms, cudaStream_t s);

template <class VT>
struct Step1Args {
  int NN, iter;
  double dt;
  const int *k_off, *k_col;  // SELL-32
  const VT* kval;
  const int *g_off, *g_col;  // SELL-32
  const VT *g1, *g2, *g3;
  const GVec<VT>* uprev;  // UnpHalf_prev, gathered by K
  const double4 *un, *r1conv, *kacc;
  const float4* r1conv32;  // may be null: the FP32 convection term, read instead of r1conv
  const double *pn, *minv_free, *minv_orig;
  double4 *unphalf, *d, *r1out;  // r1out may be null
  GVec<VT>* unphalf_g;           // float4 copies of UnpHalf and d (VT = float)
  GVec<VT>* d_g;
};
template <class VT>
cudaError_t launch_step1(const Step1Args<VT>& a, int num_sms, cudaStream_t s);

template <class VT>
struct GtArgs {
  int NNp, pin;  // pin: row forced to 0 (< 1 disables, as the reference's node > 0 test)
  const int *gt_off, *gt_col;  // SELL-32
  const VT *gt1, *gt2, *gt3;
  const GVec<VT>* d;
  double* out;
};
template <class VT>
cudaError_t launch_gt(const GtArgs<VT>& a, int num_sms, cudaStream_t s);

template <class VT>
struct Step3Args {
  int NN, iter;
  double dt;
  const int *g_off, *g_col;  // SELL-32
  const VT *g1, *g2, *g3;
  const double* pdot;
  const double4 *kacc, *unphalf, *un, *unp1_prev;
  const double* minv_free;
  double4 *acc, *unp1, *r3out;  // r3out may be null
  double* part;                 // 3 x nblocks partials: sum U^2, sum dU^2, max |dU|/dt
  int nblocks;
  GVec<VT>* acc_g;  // float4 copy of Acc (VT = float)
};
template <class VT>
cudaError_t launch_step3(const Step3Args<VT>& a, cudaStream_t s);
int step3_blocks(int NN, int num_sms);

template <class VT>
struct SpmvK3Args {
  int NN;
  const int *off, *col;  // SELL-32
  const VT* val;
  const GVec<VT>* x;
  double4* y;
};
template <class VT>
cudaError_t launch_spmv_k3(const SpmvK3Args<VT>& a, int num_sms, cudaStream_t s);

// Pnp1 = Pn + dt*Pdot and the pressure-change partial sums.
cudaError_t launch_pressure_update(int NNp, double dt, const double* pn, const double* pdot,
                                   const double* pprev, double* pnp1, double* part, int nblocks,
                                   cudaStream_t s);
int pupdate_blocks(int NNp, int num_sms);

// out[0..4] = {sum U^2, sum dU^2, sum P^2, sum dP^2, max|dU|/dt}
cudaError_t launch_reduce_norms(const double* upart, int nub, const double* ppart, int npb, double* out,
                                cudaStream_t s);

// ---- Krylov ----
template <class VT>
struct PcgArgs {
  int n;
  const int *off, *col;  // SELL-32 Z
  const VT* val;
  const VT* dinv;
  const VT* b;
  VT* x;
  VT* work;                    // 10 n: r, u, w, z, q, s, p, n, m (two buffers)
  double* part;                // 2 x 4 x grid partial sums
  unsigned* sync;              // 1 + grid words, host-zeroed: arrival counter, block progress
  const int *nb_lo, *nb_hi;    // per block: range of blocks whose rows it gathers
  int* err;                    // host-zeroed
  double rtol;
  int maxit, warm;
  double* result;  // its, relres, status, bnorm
  unsigned long long timeout_ns;
};
// Block ranges each PCG block gathers from, for a given grid (host).
// Truncated flexible CG, FCG(m), on the SELL-32 pressure matrix (fcg.cu).
// State words in sc[]: indices below; status -1 running, 0 converged, 1
// iteration limit, 2 non-finite, 4 stalled (the residual fell by less than
// sqrt(stall2) over the last window iterations, or the direction broke
// down).  PQ0.. and Beta0.. hold (p_j, q_j) and beta_j per ring slot.
// Anchor a > 0 (with m = a + 1): directions 0..a-1 keep slots 0..a-1 for the
// whole solve and every later direction overwrites slot a, so each new
// direction is orthogonalised against the first a and the previous one.
constexpr int kFcgMaxM = 8;        // directions kept at most
constexpr int kFcgMaxBlocks = 1184;  // grid cap of the iteration kernels (8 blocks of 256 per SM on 148 SMs: one row per thread at 65^3)
enum {
  kFcgRR = 0, kFcgBB, kFcgAlpha, kFcgIt, kFcgStatus, kFcgRRMark, kFcgRtol, kFcgStall2, kFcgMaxit, kFcgWindow,
  kFcgM, kFcgAnchor, kFcgPQ0 = 12, kFcgBeta0 = kFcgPQ0 + kFcgMaxM, kFcgScalars = kFcgBeta0 + kFcgMaxM
};
// The iteration kernels read the solve's settings from sc[] (written by the
// start kernel), so a captured sequence of iterations serves every solve.
struct FcgState {
  double* sc;     // kFcgScalars words
  double* part;   // fcg_part_words(n) words
  unsigned* cnt;  // block arrival counter, zero between kernels (host-zeroed once)
  int* done;      // kernels return at once while *done != 0
  int* err;       // set when a bounded wait of the matrix stream gives up (status 3)
  unsigned long long timeout_ns;
  double rtol, stall2;  // read by the start kernel only
  int maxit, window, m;
  int anchor;  // 0: ring of the last m directions; a > 0: first a kept (m = a + 1)
};
// Slot of direction it (0-based) for window m and anchor a.
__host__ __device__ inline int fcg_slot(int it, int m, int a) {
  return a > 0 ? (it < a ? it : a) : it % m;
}
// p and q point at m ring slots of n entries each; spmv_grid: blocks of the
// SpMV kernel (two per SM, at most kFcgMaxBlocks).  stencil (may be null):
// the matrix in structured form (launch_stencil_build) on the grid fd, used
// by the SpMV instead of the SELL arrays.  z1 (may be null): the start and
// update kernels also write z1 = dinv r, the Jacobi part of the next
// preconditioned residual.
template <class VT> struct FcgArgs {
  int n; const int *off, *col; const VT* val; const VT* b;
  VT *x, *r, *z, *w, *p, *q;
  int spmv_grid;
  const VT* stencil;
  int fd[3];
  FcgState st;
  VT* z1;
  const VT* dinv;
  int pdl;  // 1: the iteration kernels launch with programmatic dependent launch
  int upd_grid;  // > 0: blocks of the update kernel (default: one thread per entry, at most kFcgMaxBlocks)
};
struct Int3 {
  int v[3];
};
// The CSR matrix (rp, col, FP64 val; identity numbering on the grid fd) in
// structured form: 125 coefficients per row, coef[slice][tap][lane] over
// 32-row slices (stencil_elems(n) entries); *bad (host-zeroed) is set when a
// coupling reaches further than two grid steps (the form does not apply).
size_t stencil_elems(int n);
template <class VT>
cudaError_t launch_stencil_build(int n, const int fd[3], const int* rp, const int* col, const double* val, VT* coef,
                                 int* bad, cudaStream_t s);
int fcg_blocks(int n);
int fcg_part_words(int n);

// Two-level preconditioner on the structured pressure grid (coarse.cu): fine
// voxel grid fd, coarse lattice cd (nc nodes), voxel -> pressure node pmap
// (null: identity), per-axis hat tables (voxel -> first coarse node i0 and
// weight f of the second), per coarse node the voxel range [lo, hi] of its
// hat along each axis, and the dense inverse of P^T Z P stored FP16 as
// inv16 = inv * inv_scale in rows of ldinv (nc rounded up to 8) entries.
template <class VT> struct CoarseArgs {
  int fd[3], cd[3], nc, ldinv;
  const int* pmap;
  const int *i0x, *i0y, *i0z;
  const double *fx, *fy, *fz;
  const int *rx, *ry, *rz;
  const __half* inv16;
  double inv_scale;
  int pdl;  // 1: the coarse kernels launch with programmatic dependent launch
};
// c = P^T r (FP32 coarse vector), e = Zc^-1 c
template <class VT>
cudaError_t launch_coarse_restrict(const CoarseArgs<VT>& a, const VT* r, float* c, const int* done, cudaStream_t s);
template <class VT>
cudaError_t launch_coarse_solve(const CoarseArgs<VT>& a, const float* c, VT* e, const int* done, cudaStream_t s);
// z[p(v)] = dinv r + (P e)[v] (e may be null) + y[v] sqrt(rr / nv) / dscale (y may be null)
template <class VT>
cudaError_t launch_precond(const CoarseArgs<VT>& a, int nv, const VT* r, const VT* dinv, const VT* e, const float* y,
                           const double* rr, double dscale, VT* z, const int* done, cudaStream_t s);
template <class VT> cudaError_t launch_fcg_start(const FcgArgs<VT>& a, int warm, cudaStream_t s);
template <class VT> cudaError_t launch_fcg_spmv(const FcgArgs<VT>& a, cudaStream_t s);
template <class VT> cudaError_t launch_fcg_update(const FcgArgs<VT>& a, cudaStream_t s);
// The two-level iteration split so that the coarse solve overlaps the SpMV
// (identity numbering, structured Z):
//   w = Z z1                               launch_fcg_spmv_jacobi (z1 from
//                                          the update), beside
//   c = P^T r, e = Zc^-1 c                 launch_coarse_restrict / _solve
//   z = z1 + P e, w += (Z P) e, dots,      launch_fcg_combine
//   coefficients
// wst: Z P per 32-row slice, 27 taps per row (wst[slice][tap][lane], tap
// dx + 3 dy + 9 dz over the row's coarse box with origin wlo[row]); e must
// hold 2 + 2 cd[0] + 2 cd[0] cd[1] zeros past its nc entries.
size_t zp_elems(int n);
template <class VT> cudaError_t launch_fcg_spmv_jacobi(const FcgArgs<VT>& a, cudaStream_t s);
template <class VT>
cudaError_t launch_fcg_combine(const FcgArgs<VT>& a, const CoarseArgs<VT>& ca, const float* wst, const int* wlo,
                               const VT* e, cudaStream_t s);

// Persistent two-level flexible CG (fcg_persist.cu): the remaining
// iterations of an FP32 inner solve that the start kernel (and any network
// iterations) began, in one cooperative launch, for an identity-numbered
// structured grid with the structured form of Z and the coarse space; m
// (the direction window) at most 4.  The solve's state words are read from
// and written back to a.st.sc; a.dinv is the FP32 Jacobi diagonal.
struct Fcg2lArgs {
  float* c;                  // coarse restriction, nc entries
  float* e;                  // coarse solution in pieces (pieces x nc partial sums)
  unsigned* sync;            // 1 + grid words, zeroed before each launch: arrival counter, block progress
  const int *nb_lo, *nb_hi;  // per block: first and last block owning a row its SpMV gathers
  double* part;              // 2 x fcg2l_part_words / 2 partial sums
  double* timing;            // may be null: 7 phase times (ns) of block 0 added per launch
  double* tblock;            // may be null: per block, the time (ns) of its SpMV phases added up
  int pieces;                // fcg2l_pieces(ldinv): e holds pieces x nc partial products
};
// Pieces per row of the coarse inverse in the coarse solve (1, 2 or 4; 0:
// the row buffers do not fit and the persistent iteration does not apply).
int fcg2l_pieces(int ldinv);
size_t fcg2l_smem_bytes();
int fcg2l_grid(int device);                                    // co-resident blocks of the launch
inline int fcg2l_part_words(int grid) { return 2 * (2 + 2 * 4) * grid; }
// blocks each block waits for: rows within `reach` of its own
void fcg2l_neighbor_ranges(int n, int grid, int reach, int* lo, int* hi);
cudaError_t launch_fcg2l(const FcgArgs<float>& a, const CoarseArgs<float>& ca, const Fcg2lArgs& pa, int grid,
                         cudaStream_t s);

// Galerkin coarse matrix on the device (galerkin.cu): W = Z P in 27-tap
// boxes and Zc = P^T W, dense and symmetrised, summed in the host build's
// order (bit-identical to coarse_build on an identity-numbered grid).
struct GalerkinArgs {
  int fd[3], cd[3];                // voxel grid, coarse lattice
  int np, nc;                      // pressure rows, coarse nodes
  const int *i0x, *i0y, *i0z;      // hat tables per axis (fd entries)
  const double *fx, *fy, *fz;
  const int *rx, *ry, *rz;         // per coarse node: first and last fine index of its support
  const int *rp, *col;             // Z in CSR (pressure numbering)
  const double* val;
  const int* vox;                  // pressure node -> voxel (null: identity)
  const int* pofv;                 // voxel -> pressure node (null: identity)
  double* w27;                     // np x 27 work: W row by row
  int* wlo;                        // np: coarse index of each row's box origin
  float* zp;                       // may be null: W in FP32, 32-row slices (split iteration)
  int* bad;                        // set when some row's box is wider than 3 nodes
  double* zc;                      // nc rows of ld doubles (zeroed by the launch)
  int ld;
};
cudaError_t launch_galerkin(const GalerkinArgs& g, cudaStream_t s);

// CSR patterns on the device (patterns.cu).  Node -> element incidence:
// counts, then (after an exclusive prefix sum of the counts into pos) the
// element of every ltog entry at pos[node]++ (order within a node arbitrary).
cudaError_t launch_incidence_count(long long nent, const int* ltog, int* cnt, cudaStream_t s);
cudaError_t launch_incidence_fill(long long nent, const int* ltog, int* pos, int* inc_el, cudaStream_t s);
struct PatArgs {
  const int *ltog, *inc_rp, *inc_el;  // element map, node -> element incidence
  const int *adj_rp, *adj_col;        // element adjacency (mode 3)
  const int* rp;                      // row pointers of the pattern written in pass 1
  int* col;                           // its columns (pass 1)
  int* len;                           // row lengths (pass 0)
  int* overflow;                      // set when a row has more candidates than a block holds
};
// mode 0: K rows (nodes of the elements around a node), 1: G rows (their
// corners), 2: element adjacency (elements sharing a node with an element),
// 3: Z rows (corners of the elements adjacent to the elements around a
// pressure node).  pass 0 writes len, pass 1 the sorted distinct columns.
cudaError_t launch_pattern_rows(const PatArgs& a, int mode, int nrows, int pass, int num_sms, cudaStream_t s);
// gt_pos[t] = index in G's columns of the entry (v, p) of G^T entry t = (p, v)
cudaError_t launch_gt_pos(int nnp, const int* gt_rp, const int* gt_col, const int* g_rp, const int* g_col, int* gt_pos,
                          int* bad, cudaStream_t s);
// first / last column of each row (0 / -1 for an empty row)
cudaError_t launch_row_ends(int n, const int* rp, const int* col, int* first, int* last, cudaStream_t s);

// Dense SPD inverse on the device (dense_chol.cu): A (row-major, leading
// dimension ld = spd_inverse_ld(n), the n x n matrix in its top-left corner)
// is replaced by its inverse; work holds ld x ld doubles; *info (device) =
// 0, or the 1-based row of the first non-positive pivot.
int spd_inverse_ld(int n);
cudaError_t spd_inverse_device(double* A, double* work, int n, int ld, int* info, cudaStream_t s);
// out (n rows of ldh halves) = inv * 16384 / max|inv| (zero past column n);
// *amax_bits receives max|inv| as the bit pattern of a double.
cudaError_t spd_inverse_to_half(const double* inv, int n, int ld, unsigned long long* amax_bits, int ldh, __half* out,
                                cudaStream_t s);

// Per block of k_pcg (grid blocks over the SELL-32 slices of n rows): the
// first and last block owning a column its slices read, from each row's
// first and last column (rows sorted ascending; last < first for an empty
// row) with the SELL padding's column 0 for empty rows.
void pcg_neighbor_ranges(int n, int grid, const int* first, const int* last, int* lo, int* hi);
template <class VT>
cudaError_t launch_pcg(const PcgArgs<VT>& a, int grid, cudaStream_t s);
template <class VT>
int pcg_max_grid(int n, int device);

// r = b - Z x (FP64, SELL-32 Z) and the partial sum of r^2 per block; rf = (float) r.
// x == null stands for x = 0 (r = b, Z is not read).
cudaError_t launch_residual64(int n, const int* off, const int* col, const double* val, const double* b,
                              const double* x, double* r, float* rf, double* part, int nblocks,
                              cudaStream_t s);
int residual_blocks(int n, int num_sms);
cudaError_t launch_axpy_f2d(int n, const float* e, double* x, cudaStream_t s);
cudaError_t launch_sum_partials(const double* part, int n, double* out, cudaStream_t s);

// CSR values -> SELL-32 values (padding entries set to 0).
template <class T>
cudaError_t launch_csr_to_sell(int nrows, const int* rp, const double* csr, const int* off, T* sell, cudaStream_t s);
// SELL-32 pattern on the device: width[s] = longest row of slice s; then,
// with off = 32 x the exclusive prefix sum of the widths (nslices + 1
// entries), the columns slice-column-major (short rows padded with their
// last column, empty rows with 0).
cudaError_t launch_sell_widths(int nrows, const int* rp, int* width, cudaStream_t s);
cudaError_t launch_sell_cols(int nrows, const int* rp, const int* col, const int* off, int* scol, cudaStream_t s);

cudaError_t launch_wait_selftest(const int* flag, int* err, unsigned long long timeout_ns, cudaStream_t s);

// layout conversion between the reference's [u|v|w] blocks and double4 nodes
cudaError_t launch_blocks_to_vec4(int NN, const double* blocks, double4* v, cudaStream_t s);
// a = b = (float4) v
cudaError_t launch_vec4_to_f32(int NN, const double4* v, float4* a, float4* b, cudaStream_t s);
cudaError_t launch_vec4_to_blocks(int NN, const double4* v, double* blocks, cudaStream_t s);
cudaError_t launch_apply_bc(int n, const int* nodes, const double* uvw, double4* u, cudaStream_t s);

}  // namespace cfd
