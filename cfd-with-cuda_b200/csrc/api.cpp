// libcfdfs C ABI: context, device buffers and the fractional-step driver.
//
// Replaces the device seam of the reference (blascoCodinaHuerta.cpp:365-377,
// CUDAcodes.cu:126-1178).  One context owns one GPU stream and every device
// buffer; nothing is allocated or freed inside the time loop (the reference
// mallocs temporaries in step2GPU and checkConvergenceGPU on every call).
// State rotation between sub-iterations and time steps swaps buffer
// pointers instead of copying (blascoCodinaHuerta.cpp:2929-2932, 3070-3071).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cfdfs.h"
#include "cuda/kernels.h"
#include "cuda/unet.h"
#include "host/coarse.h"
#include "host/problem.h"
#include "host/unet_net.h"

namespace cfd {
int make_basis(int ngp, Basis& B);
int write_tecplot(const HostProblem& P, const double* U, const double* Pn, const std::string& path,
                  const std::string& title);
int read_restart(const HostProblem& P, const std::string& path, double* U, double* Pn);
}  // namespace cfd

using namespace cfd;

struct cfd_unet {
  UnetNet net;
};

namespace {
constexpr int kFcgBatch = 4;  // flexible-CG iterations per captured graph
// An instantiated graph of kFcgBatch flexible-CG iterations and the buffers
// and network state it was captured with.
struct FcgGraph {
  struct Key {
    const void *b, *x, *work;
    const cfd_unet* net;
    int gen, plan_gen;
    bool tc;
    const int* pmap;
    const void* dinv;
    double dscale;
    int n;
    int coarse_gen;  // 0: no coarse space
    int iters;       // flexible-CG iterations in the graph
    int m;           // directions kept (selects the SpMV's instantiation)
    bool operator==(const Key& o) const {
      return b == o.b && x == o.x && work == o.work && net == o.net && gen == o.gen && plan_gen == o.plan_gen &&
             tc == o.tc && pmap == o.pmap && dinv == o.dinv && dscale == o.dscale && n == o.n &&
             coarse_gen == o.coarse_gen && iters == o.iters && m == o.m;
    }
  } key{};
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
  ~FcgGraph() { reset(); }
};
}  // namespace

namespace {

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    reset();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    n = count;
    return cudaSuccess;
  }
  size_t bytes() const { return n * sizeof(T); }
};

}  // namespace

struct cfd_ctx {
  int device = 0, num_sms = 148;
  cudaStream_t stream = nullptr;
  cfd_options opt{};
  std::string err;
  HostProblem P;
  bool loaded = false, assembled = false;

  // mesh
  DevBuf<int> ltog, bcnodes;
  DevBuf<int> elist;           // elements colour by colour (deterministic mode)
  std::vector<int> color_off;  // colour c owns elist[color_off[c] .. color_off[c+1]); empty: > 64 colours
  DevBuf<double> coord, bcvals;
  DevBuf<Basis> basis;
  DevBuf<unsigned char> bcmask;
  // patterns
  DevBuf<int> k_rp, k_col, g_rp, g_col, gt_rp, gt_col, gt_pos, z_rp, z_col;
  // FP64 operators
  DevBuf<double> kval, g1, g2, g3, gt1, gt2, gt3, zval, zdiag, zdinv, msum, minv_orig, minv_free;
  // SELL-32 copies used by the per-step kernels: layout, FP64 values and
  // (CFD_MIXED) FP32 values
  DevBuf<int> ks_off, ks_col, gs_off, gs_col, gts_off, gts_col, zs_off, zs_col;
  DevBuf<double> ks_val, gs1, gs2, gs3, gts1, gts2, gts3, zs_val;
  DevBuf<float> ks_val32, gs1_32, gs2_32, gs3_32, gts1_32, gts2_32, gts3_32, zs_val32, zdinv32;
  // velocity-sized state, double4 per node
  DevBuf<double4> vbuf[12];
  // CFD_MIXED: float4 copies of the gathered velocity vectors (Un,
  // UnpHalf_prev, UnpHalf, Acc_prev, Acc, d)
  DevBuf<float4> fbuf[7];
  float4* r1c32 = nullptr;  // CFD_MIXED: the convection term accumulated in FP32
  float4 *un32 = nullptr, *uphp32 = nullptr, *uph32 = nullptr, *accp32 = nullptr, *acc32 = nullptr,
         *d32 = nullptr;
  double4 *un = nullptr, *unp1 = nullptr, *unp1_prev = nullptr, *unphalf = nullptr, *unphalf_prev = nullptr,
          *acc = nullptr, *acc_prev = nullptr, *kacc = nullptr, *r1conv = nullptr, *dvec = nullptr, *r1dbg = nullptr,
          *r3dbg = nullptr;
  // pressure-sized state
  DevBuf<double> pbuf[6];
  double *pn = nullptr, *pnp1 = nullptr, *pnp1_prev = nullptr, *pdot = nullptr, *r2 = nullptr, *pzero = nullptr;
  // Krylov work
  DevBuf<double> cg_work, cg_part, cg_res, ir_r, ir_part, ir_sum;
  DevBuf<float> f_b, f_x, f_work;
  DevBuf<unsigned> cg_sync;
  DevBuf<int> nb64, nb32;  // per PCG block: [lo..., hi...] neighbour block ranges
  DevBuf<int> cg_err;
  int pcg_grid64 = 1, pcg_grid32 = 1, res_blocks = 1;
  // reductions
  DevBuf<double> upart, ppart, norms, blk;
  int nub = 1, npb = 1;
  double* h_small = nullptr;  // pinned scratch for small readbacks (64 doubles)

  // learned preconditioner: attached network, its grid and flexible-CG state
  cfd_unet* unet = nullptr;
  std::unique_ptr<cfd_unet> unet_owned;
  int udims[3] = {0, 0, 0};
  DevBuf<int> upmap;  // voxel -> pressure node (empty: identity)
  DevBuf<double> fcg_sc, fcg_part, fcg_work64;
  DevBuf<float> fcg_work32;
  DevBuf<float> fcg_z1;  // D^-1 r of the split FP32 iteration
  // Z P per 32-row slice, 27 taps per row, and each row's coarse box origin
  // (split FP32 iteration; cs_zp_ok when every box fits 3 x 3 x 3)
  DevBuf<float> cs_zp;
  DevBuf<int> cs_wlo;
  bool cs_zp_ok = false;
  cudaStream_t stream2 = nullptr;  // the coarse solve beside the SpMV
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  DevBuf<unsigned> fcg_cnt;
  DevBuf<int> fcg_done, fcg_err;
  int fcg_window = 25;
  bool fcg_use_graph = true;
  // CFD_FCG_SPLIT=1: the split FP32 iteration (coarse solve on a second
  // stream beside the SpMV); measured slower than the sequential form on the
  // 64^3 cavity (8.97 against 8.13 ms per step), so off by default
  bool fcg_split = false;
  // mixed-precision convection on the tensor cores (k_convect_tc) where it
  // applies; conv_err is its bounded-wait error word
  bool convect_tc = false;
  bool convect_tc_ran = false;
  DevBuf<int> conv_err;
  // CFD_FCG_ANCHOR=0: with the network in the head iterations only, keep the
  // ring of the last fcg_m directions instead of anchoring the head's
  bool fcg_anchor = true;
  // blocks per SM of the split iteration's SpMV (CFD_SPLIT_SPMV_PER_SM, 1 or
  // 2): one leaves half of every SM to the coarse kernels beside it
  int split_spmv_per_sm = 2;
  // [FP32 inner solves, FP64 solves][two-level only, with the network]
  // [window m = 1, m > 1]: the first inner solve of a mixed pressure solve
  // keeps the network's directions and the refinement solves do not, so
  // each window has its own graph instead of a re-capture per solve
  FcgGraph fcg_graph[2][2][2];
  void reset_fcg_graphs() {
    for (auto& gp : fcg_graph)
      for (auto& gq : gp)
        for (auto& g : gq) g.reset();
  }
  // CFD_FCG_PERSIST=1: the persistent two-level iteration (fcg_persist.cu)
  // for the FP32 inner solves on a structured grid instead of the per-kernel
  // iteration graphs; measured slower on the 64^3 cavity (about 85 against
  // 66 us per iteration: its grid-wide waits and serial small phases cost
  // more than the launches they replace), so off by default
  bool fcg_persist = false;
  // CFD_COARSE_HOST=1: factor and invert the coarse matrix on the host
  bool coarse_on_host = false;
  // CFD_PDL=1: the flexible-CG iteration kernels use programmatic dependent
  // launch (each may start while the one before it drains)
  bool pdl = false;
  // CFD_L2_PERSIST=1: a persisting L2 window over the coarse inverse
  bool l2_persist = false, l2_window = false;
  // CFD_COARSE_SPACING=<s>: coarse-lattice spacing in voxels (default 4)
  double coarse_spacing = 4.0;
  int fcg2l_g = 0;                  // co-resident blocks of the launch
  int fcg2l_key[3] = {0, 0, 0};     // n, blocks, reach of the neighbour ranges in fcg2l_nb
  DevBuf<unsigned> fcg2l_sync;      // arrival counter + per-block progress
  DevBuf<int> fcg2l_nb;             // [lo (blocks), hi (blocks)]
  DevBuf<double> fcg2l_part, fcg2l_time;  // time: 7 phases of block 0, then one SpMV total per block
  DevBuf<float> fcg2l_e;                   // coarse solution in pieces
  double unet_dscale = 1.0;  // median diagonal of Z (scale of the network's targets)
  double fcg_stall = 0.5;  // minimum residual reduction per window

  // structured pressure grid (udims, upmap above) and the coarse space of
  // the two-level preconditioners
  bool grid_set = false;
  std::vector<int> h_pmap;  // voxel -> pressure node (empty: identity)
  std::vector<int> h_zfirst, h_zlast;  // first / last column of each row of Z
  bool coarse_ready = false;
  int coarse_gen = 0;  // bumped on every rebuild (captured graphs key on it)
  int cs_fd[3] = {0, 0, 0}, cs_cd[3] = {0, 0, 0}, cs_nc = 0;
  DevBuf<int> cs_i0[3], cs_r[3];
  DevBuf<double> cs_f[3], cs_e64;
  DevBuf<float> cs_c32, cs_e32;  // coarse right-hand side (both precisions), FP32 coarse solution
  DevBuf<__half> cs_inv16;

  // blocks of the flexible-CG update kernel, four entries per thread:
  // 4 per SM by default (fewer partial sums for the last block to add than
  // one thread per entry; 131.5 against 127.9 steps/s on the 64^3 two-level
  // line); CFD_FCG_UPDATE_BLOCKS overrides it, 0 = one thread per entry
  int upd_grid = -1;
  // CFD_HOST_PATTERNS=1: the CSR patterns are built on the host (the
  // fallback of the device build)
  bool host_patterns = false;
  DevBuf<float> zst32;  // Z in structured (125-tap) form for the FP32 inner solves, when it applies
  bool zst_ok = false;
  int cs_ld = 0;
  double cs_scale = 1.0;
  double coarse_setup_s = 0;

  int timeN = 0;
  double timeT = 0, maxAcc = 0;
  // set by cfd_rotate, cleared by cfd_step3 and cfd_begin_step: the latest
  // Unp1 / Pnp1 then sit in the _prev buffers
  bool rotated = false;
  double last_norms[5] = {0, 0, 0, 0, 0};
  bool r_debug = true;

  // launch counting and per-kernel-class event timing
  long long launches = 0;
  bool prof_on = false;
  struct Pair {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<cudaEvent_t> ev_pool;
  std::vector<Pair> pending;
  double prof[CFD_K_COUNT][3] = {};
  ~cfd_ctx() {
    for (auto& p : pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    for (auto e : ev_pool) cudaEventDestroy(e);
  }
};

namespace {

int fail(cfd_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CU(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(c, e_ == cudaErrorMemoryAllocation ? CFD_E_NOMEM : CFD_E_CUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                            \
  } while (0)

#define NEED(cond, msg)                                                        \
  do {                                                                         \
    if (!(cond)) return fail(c, CFD_E_BADARG, "%s", msg);                      \
  } while (0)

template <class T>
cudaError_t upload(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
  cudaError_t e = d.alloc(h.size());
  if (e != cudaSuccess) return e;
  if (h.empty()) return cudaSuccess;
  return cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

// SELL-32 copy of a CSR pattern already on the device: slice widths on the
// device, their prefix sum on the host (nrows / 32 entries), the padded
// columns on the device.  entries = stored entries (slices x 32 x width).
int sell_pattern(cfd_ctx* c, int nrows, const int* rp, const int* col, DevBuf<int>& off, DevBuf<int>& scol,
                 size_t& entries) {
  const int ns = (nrows + 31) / 32;
  DevBuf<int> width;
  CU(width.alloc(ns));
  CU(launch_sell_widths(nrows, rp, width.p, c->stream));
  std::vector<int> w(ns), h(ns + 1, 0);
  CU(cudaMemcpyAsync(w.data(), width.p, ns * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  long long total = 0;
  for (int i = 0; i < ns; i++) {
    total += 32LL * w[i];
    if (total >= (1LL << 31)) return fail(c, CFD_E_BADINPUT, "an operator exceeds 2^31 stored entries");
    h[i + 1] = (int)total;
  }
  CU(upload(off, h, c->stream));
  CU(scol.alloc((size_t)total));
  CU(launch_sell_cols(nrows, rp, col, off.p, scol.p, c->stream));
  entries = (size_t)total;
  return CFD_OK;
}

// Exclusive prefix sum of n counts into n + 1 row pointers (host);
// false when the total reaches 2^31.
bool row_pointers(const std::vector<int>& len, std::vector<int>& rp, int& maxlen) {
  rp.assign(len.size() + 1, 0);
  long long t = 0;
  maxlen = 0;
  for (size_t i = 0; i < len.size(); i++) {
    t += len[i];
    if (t >= (1LL << 31) - 1) return false;
    rp[i + 1] = (int)t;
    maxlen = std::max(maxlen, len[i]);
  }
  return true;
}

// The CSR patterns of K, G, G^T (with gt_pos) and Z built on the device from
// the uploaded element map (patterns.cu), with the row pointers kept on the
// host too (P.k_rp ...; the columns stay on the device until
// ensure_host_columns).  built = false, with nothing changed, when a row has
// more candidates than the device build holds: the caller builds them on the
// host.
int device_patterns(cfd_ctx* c, bool& built) {
  built = false;
  HostProblem& P = c->P;
  cudaStream_t s = c->stream;
  const int NN = P.NN, NNp = P.NNp, NE = P.NE;
  const long long nent = 27LL * NE;
  DevBuf<int> cnt, inc_rp, inc_el, pos, len, flag, adj_rp, adj_col;
  CU(cnt.alloc(NN));
  CU(cudaMemsetAsync(cnt.p, 0, (size_t)NN * sizeof(int), s));
  CU(launch_incidence_count(nent, c->ltog.p, cnt.p, s));
  std::vector<int> h(NN), hrp;
  CU(cudaMemcpyAsync(h.data(), cnt.p, (size_t)NN * sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  int maxdeg = 0;
  if (!row_pointers(h, hrp, maxdeg)) return fail(c, CFD_E_BADINPUT, "element map too large");
  CU(upload(inc_rp, hrp, s));
  CU(upload(pos, hrp, s));
  CU(inc_el.alloc((size_t)nent));
  CU(launch_incidence_fill(nent, c->ltog.p, pos.p, inc_el.p, s));
  CU(flag.alloc(1));
  CU(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  CU(len.alloc(std::max(NN, NE)));
  PatArgs a{};
  a.ltog = c->ltog.p;
  a.inc_rp = inc_rp.p;
  a.inc_el = inc_el.p;
  a.len = len.p;
  a.overflow = flag.p;
  // one pattern: pass 0 (lengths), host row pointers, pass 1 (columns)
  auto one = [&](int mode, int nrows, DevBuf<int>& drp, DevBuf<int>& dcol, std::vector<int>& rp, int& maxlen,
                 bool& ok) -> int {
    ok = false;
    a.rp = nullptr;
    a.col = nullptr;
    CU(launch_pattern_rows(a, mode, nrows, 0, c->num_sms, s));
    std::vector<int> hl(nrows);
    int hf = 0;
    CU(cudaMemcpyAsync(hl.data(), len.p, (size_t)nrows * sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&hf, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (hf) return CFD_OK;
    if (!row_pointers(hl, rp, maxlen)) return fail(c, CFD_E_BADINPUT, "an operator has more than 2^31 non-zeros");
    CU(upload(drp, rp, s));
    CU(dcol.alloc((size_t)rp[nrows]));
    a.rp = drp.p;
    a.col = dcol.p;
    CU(launch_pattern_rows(a, mode, nrows, 1, c->num_sms, s));
    ok = true;
    return CFD_OK;
  };
  bool ok = false;
  std::vector<int> k_rp, g_rp, z_rp, adj_h;
  int maxK = 0, maxG = 0, maxZ = 0, maxA = 0;
  int rc = one(0, NN, c->k_rp, c->k_col, k_rp, maxK, ok);
  if (rc || !ok) return rc;
  rc = one(1, NN, c->g_rp, c->g_col, g_rp, maxG, ok);
  if (rc || !ok) return rc;
  rc = one(2, NE, adj_rp, adj_col, adj_h, maxA, ok);
  if (rc || !ok) return rc;
  a.adj_rp = adj_rp.p;
  a.adj_col = adj_col.p;
  rc = one(3, NNp, c->z_rp, c->z_col, z_rp, maxZ, ok);
  if (rc || !ok) return rc;
  // G^T is K's first NNp rows (pressure nodes are the corner nodes 0 .. NNp)
  const long long nnzG = g_rp[NN], nnzGt = k_rp[NNp];
  if (nnzGt != nnzG) return fail(c, CFD_E_BADINPUT, "inconsistent G and G^T patterns");
  std::vector<int> gt_rp(k_rp.begin(), k_rp.begin() + NNp + 1);
  CU(upload(c->gt_rp, gt_rp, s));
  CU(c->gt_col.alloc((size_t)nnzG));
  CU(cudaMemcpyAsync(c->gt_col.p, c->k_col.p, (size_t)nnzG * sizeof(int), cudaMemcpyDeviceToDevice, s));
  CU(c->gt_pos.alloc((size_t)nnzG));
  CU(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  CU(launch_gt_pos(NNp, c->gt_rp.p, c->gt_col.p, c->g_rp.p, c->g_col.p, c->gt_pos.p, flag.p, s));
  // first / last column of Z's rows (the k_pcg neighbour ranges)
  DevBuf<int> zf, zl;
  CU(zf.alloc(NNp));
  CU(zl.alloc(NNp));
  CU(launch_row_ends(NNp, c->z_rp.p, c->z_col.p, zf.p, zl.p, s));
  c->h_zfirst.resize(NNp);
  c->h_zlast.resize(NNp);
  int hbad = 0;
  CU(cudaMemcpyAsync(c->h_zfirst.data(), zf.p, (size_t)NNp * sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(c->h_zlast.data(), zl.p, (size_t)NNp * sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(&hbad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (hbad) return fail(c, CFD_E_BADINPUT, "inconsistent G and G^T patterns");
  int maxGt = 0;
  for (int r = 0; r < NNp; r++) maxGt = std::max(maxGt, k_rp[r + 1] - k_rp[r]);
  P.k_rp.swap(k_rp);
  P.g_rp.swap(g_rp);
  P.gt_rp.swap(gt_rp);
  P.z_rp.swap(z_rp);
  P.k_col.clear();
  P.g_col.clear();
  P.gt_col.clear();
  P.gt_pos.clear();
  P.z_col.clear();
  P.maxKrow = maxK;
  P.maxGrow = maxG;
  P.maxGtrow = maxGt;
  P.maxZrow = maxZ;
  P.nnzK = P.k_rp[NN];
  P.nnzG = nnzG;
  P.nnzZ = P.z_rp[NNp];
  built = true;
  return CFD_OK;
}

// The host copies of the pattern columns, downloaded from the device when the
// patterns were built there (for cfd_download_matrix and the host build of
// the coarse space).
int ensure_host_columns(cfd_ctx* c) {
  HostProblem& P = c->P;
  if (!P.k_col.empty() || P.nnzK == 0) return CFD_OK;
  P.k_col.resize((size_t)P.nnzK);
  P.g_col.resize((size_t)P.nnzG);
  P.gt_col.resize((size_t)P.nnzG);
  P.gt_pos.resize((size_t)P.nnzG);
  P.z_col.resize((size_t)P.nnzZ);
  CU(cudaStreamSynchronize(c->stream));
  CU(cudaMemcpy(P.k_col.data(), c->k_col.p, P.k_col.size() * sizeof(int), cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(P.g_col.data(), c->g_col.p, P.g_col.size() * sizeof(int), cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(P.gt_col.data(), c->gt_col.p, P.gt_col.size() * sizeof(int), cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(P.gt_pos.data(), c->gt_pos.p, P.gt_pos.size() * sizeof(int), cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(P.z_col.data(), c->z_col.p, P.z_col.size() * sizeof(int), cudaMemcpyDeviceToHost));
  return CFD_OK;
}

int set_device(cfd_ctx* c) {
  CU(cudaSetDevice(c->device));
  return CFD_OK;
}

double wall_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool mixed(const cfd_ctx* c);

cudaEvent_t take_event(cfd_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Converts finished event pairs into per-class totals (call after a sync).
void harvest(cfd_ctx* c) {
  for (auto& p : c->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      c->prof[p.cls][0] += 1;
      c->prof[p.cls][1] += ms;
    }
    c->ev_pool.push_back(p.a);
    c->ev_pool.push_back(p.b);
  }
  c->pending.clear();
}

// Issues one kernel launch on the context stream, counting it and, when
// profiling is on, bracketing it with CUDA events.
template <class F>
int klaunch(cfd_ctx* c, int cls, F&& f) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (c->prof_on) {
    a = take_event(c);
    b = take_event(c);
    cudaEventRecord(a, c->stream);
  }
  cudaError_t e = f();
  c->launches++;
  if (c->prof_on) {
    cudaEventRecord(b, c->stream);
    c->pending.push_back({cls, a, b});
  }
  if (e != cudaSuccess)
    return fail(c, e == cudaErrorMemoryAllocation ? CFD_E_NOMEM : CFD_E_CUDA, "kernel launch (class %d): %s", cls,
                cudaGetErrorString(e));
  return CFD_OK;
}

#define KL(cls, expr)                                           \
  do {                                                          \
    int rc_ = klaunch(c, cls, [&]() { return (expr); });        \
    if (rc_) return rc_;                                        \
  } while (0)

// Allocates every device buffer and uploads mesh, patterns, BC data and the
// initial condition (initializeAndAllocateGPU, CUDAcodes.cu:161-274, and
// applyBC_initial, blascoCodinaHuerta.cpp:4062-4110).
int upload_problem(cfd_ctx* c) {
  HostProblem& P = c->P;
  cudaStream_t s = c->stream;
  if (c->opt.ngp_override) P.NGP = c->opt.ngp_override;
  Basis hb;
  if (make_basis(P.NGP, hb)) return fail(c, CFD_E_BADINPUT, "unsupported NGP %d", P.NGP);
  CU(c->basis.alloc(1));
  CU(cudaMemcpyAsync(c->basis.p, &hb, sizeof(Basis), cudaMemcpyHostToDevice, s));
  CU(upload(c->ltog, P.ltog, s));
  CU(upload(c->coord, P.coord, s));
  {
    std::vector<int> order;
    c->color_off.clear();
    if (color_elements(P, order, c->color_off) == 0) {
      CU(upload(c->elist, order, s));
    } else {
      c->color_off.clear();
    }
  }
  // CSR patterns: built on the device unless the host already has them (or
  // a row exceeds what the device build holds)
  bool on_device = false;
  if (P.k_rp.empty()) {
    int rc = c->host_patterns ? CFD_OK : device_patterns(c, on_device);
    if (rc) return rc;
    if (!on_device) {
      rc = build_patterns(P, c->err);
      if (rc) return rc;
    }
  }
  if (!on_device) {
    CU(upload(c->k_rp, P.k_rp, s));
    CU(upload(c->k_col, P.k_col, s));
    CU(upload(c->g_rp, P.g_rp, s));
    CU(upload(c->g_col, P.g_col, s));
    CU(upload(c->gt_rp, P.gt_rp, s));
    CU(upload(c->gt_col, P.gt_col, s));
    CU(upload(c->gt_pos, P.gt_pos, s));
    CU(upload(c->z_rp, P.z_rp, s));
    CU(upload(c->z_col, P.z_col, s));
    c->h_zfirst.resize(P.NNp);
    c->h_zlast.resize(P.NNp);
    for (int r = 0; r < P.NNp; r++) {
      const int b = P.z_rp[r], e = P.z_rp[r + 1];
      c->h_zfirst[r] = b < e ? P.z_col[b] : 0;
      c->h_zlast[r] = b < e ? P.z_col[e - 1] : -1;
    }
  }
  // SELL-32 copies of the patterns, built on the device
  size_t sK = 0, sG = 0, sGt = 0, sZ = 0;
  {
    int rc = sell_pattern(c, (int)P.NN, c->k_rp.p, c->k_col.p, c->ks_off, c->ks_col, sK);
    if (!rc) rc = sell_pattern(c, (int)P.NN, c->g_rp.p, c->g_col.p, c->gs_off, c->gs_col, sG);
    if (!rc) rc = sell_pattern(c, (int)P.NNp, c->gt_rp.p, c->gt_col.p, c->gts_off, c->gts_col, sGt);
    if (!rc) rc = sell_pattern(c, (int)P.NNp, c->z_rp.p, c->z_col.p, c->zs_off, c->zs_col, sZ);
    if (rc) return rc;
  }
  std::vector<unsigned char> mask(P.NN, 0);
  std::vector<double> bcv(3 * P.bcnode.size());
  for (size_t i = 0; i < P.bcnode.size(); i++) {
    mask[P.bcnode[i]] = 1;
    for (int d = 0; d < 3; d++) bcv[3 * i + d] = P.bcstr[3 * (size_t)P.bcid[i] + d];
  }
  CU(upload(c->bcmask, mask, s));
  CU(upload(c->bcnodes, P.bcnode, s));
  CU(upload(c->bcvals, bcv, s));
  const size_t NN = P.NN, NNp = P.NNp;
  const size_t nnzK = (size_t)P.nnzK, nnzG = (size_t)P.nnzG, nnzZ = (size_t)P.nnzZ;
  for (auto* b : {&c->kval}) CU(b->alloc(nnzK));
  for (auto* b : {&c->g1, &c->g2, &c->g3, &c->gt1, &c->gt2, &c->gt3}) CU(b->alloc(nnzG));
  CU(c->zval.alloc(nnzZ));
  for (auto* b : {&c->zdiag, &c->zdinv}) CU(b->alloc(NNp));
  for (auto* b : {&c->msum, &c->minv_orig, &c->minv_free}) CU(b->alloc(NN));
  CU(c->ks_val.alloc(sK));
  for (auto* b : {&c->gs1, &c->gs2, &c->gs3}) CU(b->alloc(sG));
  for (auto* b : {&c->gts1, &c->gts2, &c->gts3}) CU(b->alloc(sGt));
  CU(c->zs_val.alloc(sZ));
  if (c->opt.precision == CFD_MIXED) {
    CU(c->ks_val32.alloc(sK));
    for (auto* b : {&c->gs1_32, &c->gs2_32, &c->gs3_32}) CU(b->alloc(sG));
    for (auto* b : {&c->gts1_32, &c->gts2_32, &c->gts3_32}) CU(b->alloc(sGt));
    CU(c->zs_val32.alloc(sZ));
    CU(c->zdinv32.alloc(NNp));
    for (auto* b : {&c->f_b, &c->f_x}) CU(b->alloc(NNp));
    CU(c->f_work.alloc(10 * NNp));
  }
  for (auto& b : c->vbuf) {
    CU(b.alloc(NN));
    CU(cudaMemsetAsync(b.p, 0, b.bytes(), s));
  }
  c->un = c->vbuf[0].p; c->unp1 = c->vbuf[1].p; c->unp1_prev = c->vbuf[2].p; c->unphalf = c->vbuf[3].p;
  c->unphalf_prev = c->vbuf[4].p; c->acc = c->vbuf[5].p; c->acc_prev = c->vbuf[6].p; c->kacc = c->vbuf[7].p;
  c->r1conv = c->vbuf[8].p; c->dvec = c->vbuf[9].p; c->r1dbg = c->vbuf[10].p; c->r3dbg = c->vbuf[11].p;
  if (mixed(c)) {
    for (auto& b : c->fbuf) {
      CU(b.alloc(NN));
      CU(cudaMemsetAsync(b.p, 0, b.bytes(), s));
    }
    c->un32 = c->fbuf[0].p; c->uphp32 = c->fbuf[1].p; c->uph32 = c->fbuf[2].p;
    c->accp32 = c->fbuf[3].p; c->acc32 = c->fbuf[4].p; c->d32 = c->fbuf[5].p;
    c->r1c32 = c->fbuf[6].p;
  }
  for (auto& b : c->pbuf) {
    CU(b.alloc(NNp));
    CU(cudaMemsetAsync(b.p, 0, b.bytes(), s));
  }
  c->pn = c->pbuf[0].p; c->pnp1 = c->pbuf[1].p; c->pnp1_prev = c->pbuf[2].p; c->pdot = c->pbuf[3].p;
  c->r2 = c->pbuf[4].p; c->pzero = c->pbuf[5].p;
  CU(c->ir_r.alloc(NNp));
  CU(c->cg_work.alloc(10 * NNp));
  c->pcg_grid64 = pcg_max_grid<double>((int)NNp, c->device);
  c->pcg_grid32 = pcg_max_grid<float>((int)NNp, c->device);
  const int gmax = std::max(c->pcg_grid64, c->pcg_grid32);
  CU(c->cg_part.alloc(8 * (size_t)gmax));
  CU(c->cg_sync.alloc(1 + (size_t)gmax));
  for (int pass = 0; pass < 2; pass++) {
    const int grid = pass == 0 ? c->pcg_grid64 : c->pcg_grid32;
    std::vector<int> nb(2 * (size_t)grid);
    pcg_neighbor_ranges((int)NNp, grid, c->h_zfirst.data(), c->h_zlast.data(), nb.data(), nb.data() + grid);
    CU(upload(pass == 0 ? c->nb64 : c->nb32, nb, s));
  }
  CU(c->cg_res.alloc(8));

  CU(c->cg_err.alloc(1));
  c->res_blocks = residual_blocks((int)NNp, c->num_sms);
  CU(c->ir_part.alloc(c->res_blocks));
  CU(c->ir_sum.alloc(2));
  c->nub = step3_blocks((int)NN, c->num_sms);
  c->npb = pupdate_blocks((int)NNp, c->num_sms);
  CU(c->upart.alloc(3 * (size_t)c->nub));
  CU(c->ppart.alloc(2 * (size_t)c->npb));
  CU(cudaMemsetAsync(c->upart.p, 0, c->upart.bytes(), s));
  CU(cudaMemsetAsync(c->ppart.p, 0, c->ppart.bytes(), s));
  CU(c->norms.alloc(8));
  CU(c->blk.alloc(3 * NN));
  // initial condition: Un = BC values at Dirichlet nodes, zero elsewhere
  CU(launch_apply_bc((int)P.bcnode.size(), c->bcnodes.p, c->bcvals.p, c->un, s));
  CU(cudaStreamSynchronize(s));
  c->timeN = 0;
  c->timeT = P.t_ini;
  c->loaded = true;
  c->assembled = false;
  return CFD_OK;
}

// ---- pressure solves ----------------------------------------------------

int run_pcg64(cfd_ctx* c, const double* b, double* x, int warm, double rtol, int maxit, double* res) {
  cudaStream_t s = c->stream;
  CU(cudaMemsetAsync(c->cg_sync.p, 0, c->cg_sync.bytes(), s));
  CU(cudaMemsetAsync(c->cg_err.p, 0, sizeof(int), s));
  PcgArgs<double> a{};
  a.n = c->P.NNp;
  a.off = c->zs_off.p; a.col = c->zs_col.p; a.val = c->zs_val.p; a.dinv = c->zdinv.p;
  a.b = b; a.x = x; a.work = c->cg_work.p;
  a.part = c->cg_part.p; a.sync = c->cg_sync.p; a.err = c->cg_err.p;
  a.nb_lo = c->nb64.p; a.nb_hi = c->nb64.p + c->pcg_grid64;
  a.rtol = rtol; a.maxit = maxit; a.warm = warm; a.result = c->cg_res.p;
  a.timeout_ns = 2000000000ULL;
  KL(CFD_K_PCG64, launch_pcg<double>(a, c->pcg_grid64, s));
  CU(cudaMemcpyAsync(c->h_small, c->cg_res.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  for (int i = 0; i < 4; i++) res[i] = c->h_small[i];
  if (c->prof_on) c->prof[CFD_K_PCG64][2] += res[0];
  return CFD_OK;
}

int run_pcg32(cfd_ctx* c, double rtol, int maxit, double* res) {
  cudaStream_t s = c->stream;
  CU(cudaMemsetAsync(c->cg_sync.p, 0, c->cg_sync.bytes(), s));
  CU(cudaMemsetAsync(c->cg_err.p, 0, sizeof(int), s));
  PcgArgs<float> a{};
  a.n = c->P.NNp;
  a.off = c->zs_off.p; a.col = c->zs_col.p; a.val = c->zs_val32.p; a.dinv = c->zdinv32.p;
  a.b = c->f_b.p; a.x = c->f_x.p; a.work = c->f_work.p;
  a.part = c->cg_part.p; a.sync = c->cg_sync.p; a.err = c->cg_err.p;
  a.nb_lo = c->nb32.p; a.nb_hi = c->nb32.p + c->pcg_grid32;
  a.rtol = rtol; a.maxit = maxit; a.warm = 0; a.result = c->cg_res.p;
  a.timeout_ns = 2000000000ULL;
  KL(CFD_K_PCG32, launch_pcg<float>(a, c->pcg_grid32, s));
  CU(cudaMemcpyAsync(c->h_small, c->cg_res.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  for (int i = 0; i < 4; i++) res[i] = c->h_small[i];
  if (c->prof_on) c->prof[CFD_K_PCG32][2] += res[0];
  return CFD_OK;
}

bool learned(const cfd_ctx* c);
bool twolevel(const cfd_ctx* c);

// Voxel grid of the pressure nodes: dims, voxel -> node map (host and
// device copies; empty = identity).
int set_grid(cfd_ctx* c, const int dims[3], const int* p_of_vox) {
  const long long nv = (long long)dims[0] * dims[1] * dims[2];
  NEED(dims[0] > 0 && dims[1] > 0 && dims[2] > 0 && nv == c->P.NNp,
       "grid dims do not multiply to the number of pressure nodes");
  std::vector<int> pm;
  if (p_of_vox) {
    std::vector<char> seen(nv, 0);
    for (long long v = 0; v < nv; v++) {
      NEED(p_of_vox[v] >= 0 && p_of_vox[v] < nv && !seen[p_of_vox[v]], "p_of_vox is not a permutation");
      seen[p_of_vox[v]] = 1;
    }
    pm.assign(p_of_vox, p_of_vox + nv);
  }
  c->upmap.reset();
  if (!pm.empty()) {
    CU(c->upmap.alloc(nv));
    CU(cudaMemcpyAsync(c->upmap.p, pm.data(), nv * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CU(cudaStreamSynchronize(c->stream));
  }
  c->h_pmap = std::move(pm);
  for (int a = 0; a < 3; a++) c->udims[a] = dims[a];
  c->grid_set = true;
  c->coarse_ready = false;
  c->reset_fcg_graphs();
  return CFD_OK;
}

// Without a declared grid: a cube of m^3 pressure nodes numbered x + m (y +
// m z), accepted only if the node coordinates increase along each index.
int ensure_grid(cfd_ctx* c) {
  if (c->grid_set) return CFD_OK;
  const long long np = c->P.NNp;
  const int m = (int)std::llround(std::cbrt((double)np));
  NEED((long long)m * m * m == np && m >= 2,
       "pressure nodes do not form a cube: declare the grid with cfd_set_pressure_grid");
  const double* X = c->P.coord.data();
  for (long long v = 0; v < np; v++) {
    const int x = (int)(v % m), y = (int)((v / m) % m), z = (int)(v / ((long long)m * m));
    const bool ok = (x == 0 || X[3 * v] > X[3 * (v - 1)]) && (y == 0 || X[3 * v + 1] > X[3 * (v - m) + 1]) &&
                    (z == 0 || X[3 * v + 2] > X[3 * (v - (long long)m * m) + 2]);
    NEED(ok, "pressure nodes are not numbered x + m (y + m z): declare the grid with cfd_set_pressure_grid");
  }
  const int d[3] = {m, m, m};
  return set_grid(c, d, nullptr);
}

constexpr int kCoarseMaxNodes = 6000;

// With CFD_L2_PERSIST=1, keeps [p, p + bytes) in L2 across the kernels of
// the context's stream (and the graphs captured from it): a
// persisting-access window with an L2 set-aside of at most the device's
// limit.  The coarse inverse is read once per two-level iteration, between
// passes of the 137 MB structured-Z stream (read evict-first).  Measured on
// the 64^3 cavity's two-level line the window made the steps slower (126.5
// against 128.7 steps/s), so it is off by default.  The set-aside belongs
// to this process's context; cfd_destroy releases it.
// contexts of this process holding a persisting window (they share the
// device's CUDA context and its set-aside)
std::atomic<int> g_l2_users{0};

int keep_in_l2(cfd_ctx* c, void* p, size_t bytes) {
  if (!c->l2_persist || !p || bytes == 0) return CFD_OK;
  int maxpersist = 0, maxwin = 0;
  cudaDeviceGetAttribute(&maxpersist, cudaDevAttrMaxPersistingL2CacheSize, c->device);
  cudaDeviceGetAttribute(&maxwin, cudaDevAttrMaxAccessPolicyWindowSize, c->device);
  if (maxpersist <= 0 || maxwin <= 0) return CFD_OK;
  const size_t win = std::min(bytes, (size_t)maxwin);
  const size_t setaside = std::min(win, (size_t)maxpersist);
  CU(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, setaside));
  cudaStreamAttrValue v{};
  v.accessPolicyWindow.base_ptr = p;
  v.accessPolicyWindow.num_bytes = win;
  v.accessPolicyWindow.hitRatio = std::min(1.0f, (float)setaside / (float)win);
  v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  CU(cudaStreamSetAttribute(c->stream, cudaStreamAttributeAccessPolicyWindow, &v));
  if (!c->l2_window) g_l2_users++;
  c->l2_window = true;
  return CFD_OK;
}

// Hat functions of the coarse lattice along one axis of n fine nodes and ncd
// coarse nodes h apart: fine index x lies in coarse cell i0[x] with weight
// 1 - f[x] on node i0 and f[x] on node i0 + 1 (the tables of coarse.cpp);
// rng[2k], rng[2k + 1] = the first and last fine index in node k's support.
void hat_tables(int n, int ncd, double h, std::vector<int>& i0, std::vector<double>& f, std::vector<int>& rng) {
  i0.assign(n, 0);
  f.assign(n, 0.0);
  rng.assign(2 * (size_t)ncd, 0);
  for (int i = 0; i < ncd; i++) {
    rng[2 * i] = n;
    rng[2 * i + 1] = -1;
  }
  for (int x = 0; x < n; x++) {
    int i = 0;
    double fr = 0.0;
    if (ncd >= 2) {
      const double t = x / h;
      i = std::min(std::max((int)std::floor(t), 0), ncd - 2);
      fr = std::min(std::max(t - i, 0.0), 1.0);
    }
    i0[x] = i;
    f[x] = fr;
    for (int k = i; k <= std::min(i + 1, ncd - 1); k++) {
      rng[2 * k] = std::min(rng[2 * k], x);
      rng[2 * k + 1] = std::max(rng[2 * k + 1], x);
    }
  }
  for (int i = 0; i < ncd; i++)
    if (rng[2 * i + 1] < rng[2 * i]) rng[2 * i] = rng[2 * i + 1] = 0;
}

// Builds the coarse space from the assembled Z and puts on the device the
// hat tables and the scaled FP16 inverse of P^T Z P.
int ensure_coarse(cfd_ctx* c) {
  if (c->coarse_ready) return CFD_OK;
  int rc = ensure_grid(c);
  if (rc) return rc;
  const double t0 = wall_seconds();
  const HostProblem& P = c->P;
  const int np = P.NNp;
  CoarseSpace cs;
  for (int a = 0; a < 3; a++) cs.fd[a] = c->udims[a];
  coarse_lattice(c->udims, kCoarseMaxNodes, cs.cd, cs.h, c->coarse_spacing);
  cs.nc = cs.cd[0] * cs.cd[1] * cs.cd[2];
  const int nc = cs.nc;
  for (int a = 0; a < 3; a++) {
    c->cs_fd[a] = cs.fd[a];
    c->cs_cd[a] = cs.cd[a];
    const int n = cs.fd[a], ncd = cs.cd[a];
    std::vector<int> i0, rng;
    std::vector<double> f;
    hat_tables(n, ncd, cs.h[a], i0, f, rng);
    CU(c->cs_i0[a].alloc(n));
    CU(c->cs_f[a].alloc(n));
    CU(c->cs_r[a].alloc(2 * (size_t)ncd));
    CU(cudaMemcpy(c->cs_i0[a].p, i0.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(c->cs_f[a].p, f.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(c->cs_r[a].p, rng.data(), rng.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  c->cs_nc = nc;
  std::vector<int> vox;  // pressure node -> voxel (empty: identity)
  if (!c->h_pmap.empty()) {
    vox.assign(c->h_pmap.size(), 0);
    for (size_t v = 0; v < c->h_pmap.size(); v++) vox[c->h_pmap[v]] = (int)v;
  }
  // Z P for the split FP32 iteration (structured form, identity numbering)
  const bool want_zp = mixed(c) && c->h_pmap.empty();
  c->cs_zp_ok = false;
  c->cs_zp.reset();
  c->cs_wlo.reset();
  // The Galerkin product, the dense factorisation and the inverse of Zc run
  // on the device unless CFD_COARSE_HOST=1 keeps them on the host.  A grid
  // whose rows reach more than 3 coarse nodes per axis (a lattice finer
  // than Z's reach) builds Zc on the host and factors it on the device.
  const bool on_device = !c->coarse_on_host;
  const int ldd = spd_inverse_ld(nc);
  DevBuf<double> dA, dW;
  bool zc_on_device = false;
  if (on_device) {
    CU(dA.alloc((size_t)ldd * ldd));
    DevBuf<double> w27;
    DevBuf<int> dvox, bad, wlo;
    CU(w27.alloc(27 * (size_t)np));
    CU(bad.alloc(1));
    CU(cudaMemsetAsync(bad.p, 0, sizeof(int), c->stream));
    if (want_zp) {
      CU(c->cs_zp.alloc(zp_elems(np)));
      CU(c->cs_wlo.alloc(np));
    } else {
      CU(wlo.alloc(np));
    }
    if (!vox.empty()) {
      CU(dvox.alloc(np));
      CU(cudaMemcpyAsync(dvox.p, vox.data(), np * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    }
    GalerkinArgs g{};
    for (int a = 0; a < 3; a++) {
      g.fd[a] = cs.fd[a];
      g.cd[a] = cs.cd[a];
    }
    g.np = np;
    g.nc = nc;
    g.i0x = c->cs_i0[0].p;
    g.i0y = c->cs_i0[1].p;
    g.i0z = c->cs_i0[2].p;
    g.fx = c->cs_f[0].p;
    g.fy = c->cs_f[1].p;
    g.fz = c->cs_f[2].p;
    g.rx = c->cs_r[0].p;
    g.ry = c->cs_r[1].p;
    g.rz = c->cs_r[2].p;
    g.rp = c->z_rp.p;
    g.col = c->z_col.p;
    g.val = c->zval.p;
    g.vox = dvox.p;
    g.pofv = c->upmap.p;
    g.w27 = w27.p;
    g.wlo = want_zp ? c->cs_wlo.p : wlo.p;
    g.zp = want_zp ? c->cs_zp.p : nullptr;
    g.bad = bad.p;
    g.zc = dA.p;
    g.ld = ldd;
    CU(launch_galerkin(g, c->stream));
    int hb = 1;
    CU(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    zc_on_device = hb == 0;
    c->cs_zp_ok = zc_on_device && want_zp;
    if (!c->cs_zp_ok) {
      c->cs_zp.reset();
      c->cs_wlo.reset();
    }
  }
  if (!zc_on_device) {
    int rc = ensure_host_columns(c);
    if (rc) return rc;
    std::vector<double> zv((size_t)P.nnzZ);
    CU(cudaStreamSynchronize(c->stream));
    CU(cudaMemcpy(zv.data(), c->zval.p, zv.size() * sizeof(double), cudaMemcpyDeviceToHost));
    std::string err;
    if (coarse_build(c->udims, kCoarseMaxNodes, vox, P.z_rp, P.z_col, zv, cs, err, want_zp, !on_device,
                     c->coarse_spacing))
      return fail(c, CFD_E_NONFINITE, "%s", err.c_str());
    if (cs.nc != nc) return fail(c, CFD_E_BADARG, "coarse lattice mismatch");
    if (on_device)
      CU(cudaMemcpy2D(dA.p, ldd * sizeof(double), cs.inv.data(), nc * sizeof(double), nc * sizeof(double), nc,
                      cudaMemcpyHostToDevice));
    if (want_zp && cs.w_ok) {
      std::vector<float> zp(zp_elems(np), 0.f);
      for (int p = 0; p < np; p++)
        for (int t = 0; t < 27; t++)
          zp[((size_t)(p >> 5) * 27 + t) * 32 + (p & 31)] = (float)cs.w27[27 * (size_t)p + t];
      CU(c->cs_zp.alloc(zp.size()));
      CU(cudaMemcpy(c->cs_zp.p, zp.data(), zp.size() * sizeof(float), cudaMemcpyHostToDevice));
      CU(c->cs_wlo.alloc(np));
      CU(cudaMemcpy(c->cs_wlo.p, cs.wlo.data(), np * sizeof(int), cudaMemcpyHostToDevice));
      c->cs_zp_ok = true;
    }
  }
  // the inverse goes to the device in FP16 (rows padded to 8 entries),
  // scaled so its largest entry sits near the top of the FP16 range: the
  // coarse correction only has to be close, and halving the bytes of the
  // one dense operand of the iteration matters more
  const int ld = (nc + 7) & ~7;
  if (on_device) {
    // Cholesky and inverse in FP64, the scaled FP16 copy in place
    DevBuf<int> dinfo;
    DevBuf<unsigned long long> dmax;
    CU(dW.alloc((size_t)ldd * ldd));
    CU(dinfo.alloc(1));
    CU(dmax.alloc(1));
    CU(spd_inverse_device(dA.p, dW.p, nc, ldd, dinfo.p, c->stream));
    CU(c->cs_inv16.alloc((size_t)nc * ld));
    CU(spd_inverse_to_half(dA.p, nc, ldd, dmax.p, ld, c->cs_inv16.p, c->stream));
    int info = 0;
    unsigned long long bits = 0;
    CU(cudaMemcpyAsync(&info, dinfo.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaMemcpyAsync(&bits, dmax.p, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    if (info != 0) return fail(c, CFD_E_NONFINITE, "coarse matrix P^T Z P is not positive definite (row %d)", info);
    double amax = 0.0;
    std::memcpy(&amax, &bits, sizeof(amax));
    c->cs_scale = amax > 0 ? 16384.0 / amax : 1.0;
  } else {
    double amax = 0.0;
    for (double v : cs.inv) amax = std::max(amax, std::fabs(v));
    const double scale = amax > 0 ? 16384.0 / amax : 1.0;
    std::vector<__half> h16((size_t)nc * ld, __float2half(0.f));
    for (int i = 0; i < nc; i++)
      for (int j = 0; j < nc; j++)
        h16[(size_t)i * ld + j] = __float2half((float)(cs.inv[(size_t)i * nc + j] * scale));
    c->cs_scale = scale;
    CU(c->cs_inv16.alloc(h16.size()));
    CU(cudaMemcpy(c->cs_inv16.p, h16.data(), h16.size() * sizeof(__half), cudaMemcpyHostToDevice));
  }
  c->cs_ld = ld;
  {
    int rc = keep_in_l2(c, c->cs_inv16.p, (size_t)nc * ld * sizeof(__half));
    if (rc) return rc;
  }
  CU(c->cs_c32.alloc(ld));
  CU(cudaMemset(c->cs_c32.p, 0, ld * sizeof(float)));
  CU(c->cs_e64.alloc(nc));
  if (mixed(c)) {
    // zeros past nc: the 27-tap boxes of Z P read up to two coarse steps
    // past a row's box origin
    const size_t pad = 2 + 2 * (size_t)cs.cd[0] + 2 * (size_t)cs.cd[0] * cs.cd[1];
    CU(c->cs_e32.alloc(nc + pad));
    CU(cudaMemset(c->cs_e32.p, 0, (nc + pad) * sizeof(float)));
  }
  // FP32 inner solves on an identity-numbered grid stream Z without column
  // indices (125 coefficients per row) when every coupling stays within two
  // grid steps
  c->zst_ok = false;
  c->zst32.reset();
  if (mixed(c) && c->h_pmap.empty()) {
    DevBuf<int> bad;
    CU(bad.alloc(1));
    CU(cudaMemset(bad.p, 0, sizeof(int)));
    CU(c->zst32.alloc(stencil_elems(P.NNp)));
    CU(launch_stencil_build<float>(P.NNp, c->udims, c->z_rp.p, c->z_col.p, c->zval.p, c->zst32.p, bad.p, c->stream));
    int hb = 1;
    CU(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    c->zst_ok = hb == 0;
    if (!c->zst_ok) c->zst32.reset();
  }
  c->coarse_ready = true;
  c->coarse_gen++;
  c->reset_fcg_graphs();
  c->coarse_setup_s = wall_seconds() - t0;
  return CFD_OK;
}

template <class VT>
CoarseArgs<VT> coarse_args(const cfd_ctx* c, bool with_coarse) {
  CoarseArgs<VT> a{};
  for (int k = 0; k < 3; k++) {
    a.fd[k] = c->udims[k];
    a.cd[k] = c->cs_cd[k];
  }
  a.nc = c->cs_nc;
  a.ldinv = c->cs_ld;
  a.inv_scale = c->cs_scale;
  a.pmap = c->upmap.p;
  if (with_coarse) {
    a.i0x = c->cs_i0[0].p;
    a.i0y = c->cs_i0[1].p;
    a.i0z = c->cs_i0[2].p;
    a.fx = c->cs_f[0].p;
    a.fy = c->cs_f[1].p;
    a.fz = c->cs_f[2].p;
    a.rx = c->cs_r[0].p;
    a.ry = c->cs_r[1].p;
    a.rz = c->cs_r[2].p;
    a.inv16 = c->cs_inv16.p;
  }
  return a;
}

// Whether the persistent two-level iteration serves an FP32 solve with these
// arguments (identity-numbered structured grid with the structured form of
// Z, a window of at most 4 directions, the coarse space's limits).
bool fcg2l_fits(const cfd_ctx* c, const FcgArgs<float>& a, const CoarseArgs<float>& ca) {
  if (!c->fcg_persist || !a.stencil || ca.pmap || a.st.m < 1 || a.st.m > 4) return false;
  if ((long long)ca.fd[0] * ca.fd[1] * ca.fd[2] != a.n || ca.fd[0] > 512) return false;
  if (ca.ldinv % 8 || fcg2l_pieces(ca.ldinv) == 0) return false;
  for (int ax = 1; ax < 3; ax++) {
    const double h = ca.cd[ax] > 1 ? (double)(ca.fd[ax] - 1) / (ca.cd[ax] - 1) : 1.0;
    if ((2 * h + 1) * (2 * h + 1) > 1024) return false;
  }
  return true;
}

// The remaining iterations of an FP32 flexible-CG solve in one persistent
// launch (the start kernel and any network iterations ran before).
int run_fcg2l(cfd_ctx* c, const FcgArgs<float>& a, const CoarseArgs<float>& ca) {
  cudaStream_t s = c->stream;
  if (!c->fcg2l_g) c->fcg2l_g = fcg2l_grid(c->device);
  const int G = c->fcg2l_g;
  NEED(G > 0, "no co-resident grid for the persistent two-level iteration");
  const int reach = 2 + 2 * a.fd[0] + 2 * a.fd[0] * a.fd[1];
  if (c->fcg2l_key[0] != a.n || c->fcg2l_key[1] != G || c->fcg2l_key[2] != reach) {
    std::vector<int> nb(2 * (size_t)G);
    fcg2l_neighbor_ranges(a.n, G, reach, nb.data(), nb.data() + G);
    CU(c->fcg2l_nb.alloc(nb.size()));
    CU(cudaMemcpy(c->fcg2l_nb.p, nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice));
    CU(c->fcg2l_sync.alloc(1 + (size_t)G));
    CU(c->fcg2l_part.alloc(fcg2l_part_words(G)));
    CU(c->fcg2l_time.alloc(8 + (size_t)G));
    CU(cudaMemset(c->fcg2l_time.p, 0, (8 + (size_t)G) * sizeof(double)));
    c->fcg2l_key[0] = a.n;
    c->fcg2l_key[1] = G;
    c->fcg2l_key[2] = reach;
  }
  const int pieces = fcg2l_pieces(ca.ldinv);
  if (c->fcg2l_e.n < (size_t)pieces * ca.nc) CU(c->fcg2l_e.alloc((size_t)pieces * ca.nc));
  CU(cudaMemsetAsync(c->fcg2l_sync.p, 0, (1 + (size_t)G) * sizeof(unsigned), s));
  Fcg2lArgs pa{};
  pa.c = c->cs_c32.p;
  pa.e = c->fcg2l_e.p;
  pa.pieces = pieces;
  pa.tblock = c->prof_on ? c->fcg2l_time.p + 8 : nullptr;
  pa.sync = c->fcg2l_sync.p;
  pa.nb_lo = c->fcg2l_nb.p;
  pa.nb_hi = c->fcg2l_nb.p + G;
  pa.part = c->fcg2l_part.p;
  pa.timing = c->prof_on ? c->fcg2l_time.p : nullptr;
  KL(CFD_K_FCG2L, launch_fcg2l(a, ca, pa, G, s));
  return CFD_OK;
}

// Flexible CG with the two-level preconditioner (Jacobi step + coarse-space
// correction) and, for CFD_PC_LEARNED, the attached U-Net's correction.
// VT = float: b, x are f_b, f_x and the FP32 SELL values (inner solve of
// CFD_MIXED); VT = double: b, x are the caller's FP64 vectors.  The coarse
// space must be built (ensure_coarse) before.  res = {iterations,
// ||r||/||b||, status} with the status words of kernels.h (4 = stalled).
template <class VT>
int run_fcg(cfd_ctx* c, const VT* b, VT* x, int warm, double rtol, int maxit, double* res, bool first_solve) {
  cudaStream_t s = c->stream;
  const int n = c->P.NNp;
  // with fcg_net_iters > 0 the network serves the head of the first inner
  // solve of a pressure solve only; refinement sweeps solve for corrections
  // of a solution already accurate to the inner tolerance
  const bool use_net = learned(c) && (first_solve || c->opt.fcg_net_iters == 0);
  NEED(c->coarse_ready, "coarse space not built");
  UnetNet* netp = use_net ? &c->unet->net : nullptr;
  if (netp && netp->set_grid(c->udims, false)) return fail(c, CFD_E_NOMEM, "%s", netp->err.c_str());
  if (!c->fcg_sc.p) {
    CU(c->fcg_sc.alloc(kFcgScalars));
    CU(c->fcg_part.alloc((size_t)fcg_part_words(n)));
    CU(c->fcg_cnt.alloc(1));
    CU(cudaMemsetAsync(c->fcg_cnt.p, 0, sizeof(unsigned), s));
    CU(c->fcg_done.alloc(1));
    CU(c->fcg_err.alloc(1));
  }
  // work: r, z, w and kFcgMaxM ring slots each of p and q
  const size_t nwork = (3 + 2 * (size_t)kFcgMaxM) * n;
  FcgArgs<VT> a{};
  a.n = n;
  a.off = c->zs_off.p;
  a.col = c->zs_col.p;
  VT* work;
  if constexpr (sizeof(VT) == 4) {
    a.val = c->zs_val32.p;
    if (!c->fcg_work32.p) CU(c->fcg_work32.alloc(nwork));
    work = c->fcg_work32.p;
  } else {
    a.val = c->zs_val.p;
    if (!c->fcg_work64.p) CU(c->fcg_work64.alloc(nwork));
    work = c->fcg_work64.p;
  }
  a.b = b;
  a.x = x;
  a.r = work;
  a.z = work + (size_t)n;
  a.w = work + 2 * (size_t)n;
  a.p = work + 3 * (size_t)n;
  a.q = work + (3 + (size_t)kFcgMaxM) * n;
  a.st.sc = c->fcg_sc.p;
  a.st.part = c->fcg_part.p;
  a.st.cnt = c->fcg_cnt.p;
  a.st.done = c->fcg_done.p;
  a.st.err = c->fcg_err.p;
  a.st.timeout_ns = 2000000000ULL;
  a.spmv_grid = std::min(2 * c->num_sms, kFcgMaxBlocks);
  if constexpr (sizeof(VT) == 4) a.stencil = c->zst_ok ? c->zst32.p : nullptr;
  for (int k = 0; k < 3; k++) a.fd[k] = c->udims[k];
  a.st.rtol = rtol;
  a.st.stall2 = c->fcg_stall * c->fcg_stall;
  a.st.maxit = maxit;
  a.st.window = c->fcg_window;
  // a nonlinear (network) preconditioner needs the deeper orthogonalisation;
  // the linear two-level one is symmetric, for which FCG(1) is CG.  When
  // the network serves only the first h iterations, their directions stay
  // in slots 0..h-1 and each later one is orthogonalised against them and
  // its predecessor (m = h + 1): after the head the residual is Z-orthogonal
  // to the head's directions, and CG deflated by that space (Saad, Yeung,
  // Erhel, Guyomarc'h 2000) keeps every direction Z-orthogonal to all
  // earlier ones with this short recurrence.
  const int head_iters = c->opt.fcg_net_iters;
  const bool anchored = use_net && c->fcg_anchor && head_iters > 0 && head_iters + 1 <= kFcgMaxM;
  a.st.m = !use_net ? 1 : (anchored ? head_iters + 1 : c->opt.fcg_m);
  a.st.anchor = anchored ? head_iters : 0;
  const int* pmap = c->upmap.p;
  const VT* dinv;
  float* cc = c->cs_c32.p;
  VT* ce;
  if constexpr (sizeof(VT) == 4) {
    dinv = c->zdinv32.p;
    ce = c->cs_e32.p;
  } else {
    dinv = c->zdinv.p;
    ce = c->cs_e64.p;
  }
  // FP32 solves on the structured form with Z P available split the
  // iteration so that the coarse solve runs beside the SpMV: w = Z (D^-1 r)
  // on the solver stream, c = P^T r and e = Zc^-1 c on the second stream,
  // then z = D^-1 r + P e and w += (Z P) e with the dots (the update and
  // start kernels leave D^-1 r in z1).  Iterations with the network keep
  // the sequential form: its correction would need a second SpMV.
  const bool split = sizeof(VT) == 4 && a.stencil && c->cs_zp_ok && !pmap && c->fcg_split;
  a.dinv = dinv;
  a.pdl = c->pdl ? 1 : 0;
  a.upd_grid = c->upd_grid >= 0 ? c->upd_grid : 4 * c->num_sms;
  if (split) {
    if (!c->fcg_z1.p) CU(c->fcg_z1.alloc(n));
    a.z1 = reinterpret_cast<VT*>(c->fcg_z1.p);
  }
  KL(CFD_K_FCG, launch_fcg_start<VT>(a, warm, s));
  CoarseArgs<VT> ca = coarse_args<VT>(c, true);
  ca.pdl = a.pdl;
  // one flexible-CG iteration: preconditioner (U-Net, coarse restriction
  // and solve, combination), SpMV + dots + coefficients, update + tests
  auto iteration = [&](bool counted, bool with_net) -> int {
    UnetNet* netp_all = netp;
    UnetNet* netp = with_net ? netp_all : nullptr;
    const long long l0 = netp ? netp->launches : 0;
    auto unet = [&]() -> cudaError_t {
      cudaError_t e = unet_input(n, a.r, pmap, a.st.sc + kFcgRR, 0.0, netp->act[0], a.st.done, s);
      if (e == cudaSuccess) e = netp->forward(s, nullptr, a.st.done);
      return e;
    };
    auto coarse = [&](cudaStream_t cs) -> cudaError_t {
      cudaError_t e = launch_coarse_restrict<VT>(ca, a.r, cc, a.st.done, cs);
      if (e == cudaSuccess) e = launch_coarse_solve<VT>(ca, cc, ce, a.st.done, cs);
      return e;
    };
    auto combine = [&]() -> cudaError_t {
      return launch_precond<VT>(ca, n, a.r, dinv, ce, netp ? netp->out : nullptr, a.st.sc + kFcgRR,
                                c->unet_dscale, a.z, a.st.done, s);
    };
    if constexpr (sizeof(VT) == 4) {
      if (split && !netp) {
        // per-launch profiling times every launch on the solver stream
        const bool fork = !c->prof_on;
        cudaStream_t sb = fork ? c->stream2 : s;
        if (fork) {
          CU(cudaEventRecord(c->ev_fork, s));
          CU(cudaStreamWaitEvent(sb, c->ev_fork, 0));
        }
        FcgArgs<VT> aj = a;
        aj.spmv_grid = std::min(c->split_spmv_per_sm * c->num_sms, kFcgMaxBlocks);
        if (counted) {
          KL(CFD_K_COARSE, coarse(sb));
          KL(CFD_K_SPMV_Z, launch_fcg_spmv_jacobi<VT>(aj, s));
        } else {
          CU(coarse(sb));
          CU(launch_fcg_spmv_jacobi<VT>(aj, s));
        }
        if (fork) {
          CU(cudaEventRecord(c->ev_join, sb));
          CU(cudaStreamWaitEvent(s, c->ev_join, 0));
        }
        if (counted) {
          KL(CFD_K_FCG, launch_fcg_combine<VT>(a, ca, c->cs_zp.p, c->cs_wlo.p, ce, s));
          KL(CFD_K_FCG, launch_fcg_update<VT>(a, s));
          c->launches += 1;  // the coarse pair counts as one klaunch
        } else {
          CU(launch_fcg_combine<VT>(a, ca, c->cs_zp.p, c->cs_wlo.p, ce, s));
          CU(launch_fcg_update<VT>(a, s));
        }
        return CFD_OK;
      }
    }
    if (counted) {
      if (netp) KL(CFD_K_UNET, unet());
      KL(CFD_K_COARSE, coarse(s));
      KL(CFD_K_FCG, combine());
      KL(CFD_K_SPMV_Z, launch_fcg_spmv<VT>(a, s));
      KL(CFD_K_FCG, launch_fcg_update<VT>(a, s));
      // klaunch counted one launch for the network and one for the coarse pair
      c->launches += (netp ? netp->launches - l0 : 0) + 1;
    } else {
      if (netp) CU(unet());
      CU(coarse(s));
      CU(combine());
      CU(launch_fcg_spmv<VT>(a, s));
      CU(launch_fcg_update<VT>(a, s));
    }
    return CFD_OK;
  };
  // CUDA graphs of kFcgBatch iterations (and, when the network is applied
  // only in the first fcg_net_iters iterations, one graph of those),
  // captured once per buffer / network configuration and replayed until the
  // done flag stops the kernels
  const int net_iters = !netp ? 0 : (c->opt.fcg_net_iters > 0 ? c->opt.fcg_net_iters : 1 << 30);
  auto graph_for = [&](bool with_net, int iters, FcgGraph*& out) -> int {
    out = nullptr;
    if (!c->fcg_use_graph || c->prof_on) return CFD_OK;
    if (with_net) CU(netp->prepare_tc(s));  // packs and plans outside the capture
    FcgGraph& g = c->fcg_graph[sizeof(VT) == 4 ? 0 : 1][with_net ? 1 : 0][a.st.m > 1 ? 1 : 0];
    FcgGraph::Key key{a.b, a.x, a.r, with_net ? c->unet : nullptr, with_net ? netp->gen : 0,
                      with_net ? netp->plan_gen : 0, with_net ? netp->tc_enabled : false, pmap, dinv,
                      c->unet_dscale, n, c->coarse_gen, iters, a.st.m};
    if (!g.exec || !(g.key == key)) {
      g.reset();
      const long long l0 = with_net ? netp->launches : 0;
      CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
      int rc = CFD_OK;
      for (int k = 0; k < iters && rc == CFD_OK; k++) rc = iteration(false, with_net);
      cudaGraph_t graph = nullptr;
      cudaError_t ce = cudaStreamEndCapture(s, &graph);
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      CU(ce);
      ce = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      CU(ce);
      g.key = key;
      g.launches = (with_net ? netp->launches - l0 + iters : 0) + iters * 5;
    }
    out = &g;
    return CFD_OK;
  };
  const bool net_all = net_iters >= (1 << 30);
  const int head = net_all ? 0 : net_iters;  // iterations of the network-only head
  // after the head, the two-level iterations run in one persistent launch
  // where that applies
  bool persist = false;
  if constexpr (sizeof(VT) == 4) persist = !net_all && !split && fcg2l_fits(c, a, ca);
  FcgGraph *G = nullptr, *GH = nullptr;
  {
    int rc = persist ? CFD_OK : graph_for(net_all, kFcgBatch, G);
    if (rc) return rc;
    if (head > 0) {
      rc = graph_for(true, std::min(head, kFcgBatch), GH);
      if (rc) return rc;
    }
  }
  int issued = 0, batch = 2;
  double rr_prev = -1;
  if (head > 0) {
    // the network's iterations first, then the two-level part alone
    const int hb = std::min(head, kFcgBatch);
    for (int done_h = 0; done_h < head; done_h += hb) {
      if (GH) {
        CU(cudaGraphLaunch(GH->exec, s));
        c->launches += GH->launches;
      } else {
        for (int k = 0; k < hb; k++) {
          int rc = iteration(true, true);
          if (rc) return rc;
        }
      }
      issued += hb;
    }
  }
  if constexpr (sizeof(VT) == 4) {
    if (persist) {
      int rc = run_fcg2l(c, a, ca);
      if (rc) return rc;
      CU(cudaMemcpyAsync(c->h_small, c->fcg_sc.p, kFcgScalars * sizeof(double), cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
      if (c->prof_on) c->prof[CFD_K_FCG2L][2] += c->h_small[kFcgIt] - issued;
    }
  }
  for (; !persist;) {
    if (G) {
      const int reps = (batch + kFcgBatch - 1) / kFcgBatch;
      for (int k = 0; k < reps; k++) {
        CU(cudaGraphLaunch(G->exec, s));
        c->launches += G->launches;
      }
      batch = reps * kFcgBatch;
    } else {
      for (int k = 0; k < batch; k++) {
        int rc = iteration(true, net_all);
        if (rc) return rc;
      }
    }
    issued += batch;
    CU(cudaMemcpyAsync(c->h_small, c->fcg_sc.p, kFcgScalars * sizeof(double), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const double* h = c->h_small;
    if (h[kFcgStatus] >= 0 || issued >= maxit) break;
    // size the next batch from the observed convergence rate
    const double rr = h[kFcgRR], target = rtol * rtol * h[kFcgBB];
    int next = 4;
    if (rr_prev > 0 && rr > 0 && rr < rr_prev) {
      const double rate = std::log(rr / rr_prev) / batch;  // per iteration, < 0
      next = (int)std::ceil(std::log(target / rr) / rate);
    }
    rr_prev = rr;
    batch = std::max(1, std::min(next, 16));
  }
  const double* h = c->h_small;
  res[0] = h[kFcgIt];
  res[1] = h[kFcgBB] > 0 ? std::sqrt(h[kFcgRR] / h[kFcgBB]) : 0.0;
  res[2] = h[kFcgStatus] < 0 ? 1 : h[kFcgStatus];
  if (c->prof_on && !persist) {
    c->prof[CFD_K_FCG][2] += res[0];
    c->prof[CFD_K_SPMV_Z][2] += res[0];
  }
  return CFD_OK;
}

bool learned(const cfd_ctx* c) { return c->opt.precond == CFD_PC_LEARNED && c->unet; }
bool twolevel(const cfd_ctx* c) { return c->opt.precond == CFD_PC_TWOLEVEL; }
// solves that run flexible CG with a coarse space (and, when learned, the network)
bool fcg_path(const cfd_ctx* c) { return learned(c) || twolevel(c); }

// ||b - Z x||_2 in FP64 (also leaves r in ir_r and (float) r in f_b).
int residual_norm(cfd_ctx* c, const double* b, const double* x, double* out) {
  cudaStream_t s = c->stream;
  KL(CFD_K_RESID64, launch_residual64(c->P.NNp, c->zs_off.p, c->zs_col.p, c->zs_val.p, b, x, c->ir_r.p, c->f_b.p,
                                      c->ir_part.p, c->res_blocks, s));
  KL(CFD_K_OTHER, launch_sum_partials(c->ir_part.p, c->res_blocks, c->ir_sum.p, s));
  CU(cudaMemcpyAsync(c->h_small, c->ir_sum.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  *out = std::sqrt(c->h_small[0]);
  return CFD_OK;
}

// Solve Z x = b on the device.  FP64: one persistent Jacobi-PCG.  MIXED:
// FP64 iterative refinement around FP32 Jacobi-PCG solves (residual and
// update in FP64, inner tolerance opt.inner_rtol).
int pressure_solve(cfd_ctx* c, const double* b, double* x, int warm, cfd_solve_stats* st) {
  cfd_solve_stats z{};
  const double rtol = c->opt.cg_rtol;
  if (c->opt.precision == CFD_FP64 || c->opt.precision != CFD_MIXED) {
    double res[4] = {0, 0, 0, 0};
    int used = 0;
    if (fcg_path(c)) {
      int rc = ensure_coarse(c);
      if (rc) return rc;
      rc = run_fcg<double>(c, b, x, warm, rtol, c->opt.cg_maxit, res, true);
      if (rc) return rc;
      used = (int)res[0];
      if ((int)res[2] != 0) {
        // flexible CG stalled, broke down or ran out: Jacobi-PCG from its iterate
        z.fallback = 1;
        warm = 1;
      }
    }
    int more = 0;
    if (!fcg_path(c) || z.fallback) {
      int rc = run_pcg64(c, b, x, warm, rtol, std::max(1, c->opt.cg_maxit - used), res);
      if (rc) return rc;
      more = (int)res[0];
    }
    z.iterations = used + more;
    z.relres = res[1];
    z.status = (int)res[2];
  } else {
    cudaStream_t s = c->stream;
    if (!warm) CU(cudaMemsetAsync(x, 0, c->P.NNp * sizeof(double), s));
    double bnorm = 0, rnorm = 0;
    // ||b|| (x = 0: the residual is b itself, and f_b = b for the first inner solve)
    int rc = residual_norm(c, b, nullptr, &bnorm);
    if (rc) return rc;
    if (!std::isfinite(bnorm)) {
      z.status = 2;
    } else if (bnorm == 0.0) {
      CU(cudaMemsetAsync(x, 0, c->P.NNp * sizeof(double), s));
      z.status = 0;
    } else {
      rnorm = bnorm;
      if (warm) rc = residual_norm(c, b, x, &rnorm);
      if (rc) return rc;
      z.status = 1;
      int total = 0;
      for (int outer = 0; outer <= c->opt.max_outer; outer++) {
        if (!std::isfinite(rnorm)) { z.status = 2; break; }
        if (rnorm <= rtol * bnorm) { z.status = 0; break; }
        if (outer == c->opt.max_outer || total >= c->opt.cg_maxit) break;
        double res[4] = {0, 0, 0, 0};
        // inner target: inner_rtol relative, but no tighter than needed
        double inner = std::max(c->opt.inner_rtol, 0.5 * rtol * bnorm / rnorm);
        if (fcg_path(c) && !z.fallback) {
          rc = ensure_coarse(c);
          if (rc) return rc;
          rc = run_fcg<float>(c, c->f_b.p, c->f_x.p, 0, inner, c->opt.cg_maxit - total, res, outer == 0);
          if (rc) return rc;
          const int fs = (int)res[2];
          if (fs == 4 || fs == 2 || (fs == 1 && res[1] > 0.5)) z.fallback = 1;  // Jacobi-PCG from here on
          if (fs == 2) res[2] = 0;  // the iterate is still finite: the outer residual decides
        } else {
          rc = run_pcg32(c, inner, c->opt.cg_maxit - total, res);
          if (rc) return rc;
        }
        total += (int)res[0];
        if ((int)res[2] == 3) { z.status = 3; break; }
        KL(CFD_K_OTHER, launch_axpy_f2d(c->P.NNp, c->f_x.p, x, s));
        z.outer = outer + 1;
        rc = residual_norm(c, b, x, &rnorm);
        if (rc) return rc;
      }
      z.iterations = total;
      z.relres = rnorm / bnorm;
    }
  }
  if (st) *st = z;
  if (z.status == 3) return fail(c, CFD_E_TIMEOUT, "device-side barrier wait timed out in the pressure solve");
  if (z.status == 2) return fail(c, CFD_E_NONFINITE, "non-finite residual in the pressure solve");
  return CFD_OK;
}

int reduce_norms(cfd_ctx* c) {
  cudaStream_t s = c->stream;
  KL(CFD_K_OTHER, launch_reduce_norms(c->upart.p, c->nub, c->ppart.p, c->npb, c->norms.p, s));
  CU(cudaMemcpyAsync(c->h_small, c->norms.p, 5 * sizeof(double), cudaMemcpyDeviceToHost, s));
  int* h_conv_err = reinterpret_cast<int*>(c->h_small + 8);
  *h_conv_err = 0;
  if (c->convect_tc_ran) CU(cudaMemcpyAsync(h_conv_err, c->conv_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  for (int i = 0; i < 5; i++) c->last_norms[i] = c->h_small[i];
  if (*h_conv_err) return fail(c, CFD_E_TIMEOUT, "device-side wait timed out in the tensor-core convection");
  return CFD_OK;
}

bool mixed(const cfd_ctx* c) { return c->opt.precision == CFD_MIXED; }



}  // namespace

// =========================================================================
extern "C" {

int cfd_abi_version(void) { return CFDFS_ABI_VERSION; }

void cfd_default_options(cfd_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = CFD_FP64;
  o->precond = CFD_PC_JACOBI;
  o->cg_rtol = 1e-8;
  o->cg_maxit = 1000;
  o->cg_warm = 0;
  o->ngp_override = 0;
  o->inner_rtol = 1e-4;
  o->max_outer = 12;
  o->fcg_m = 4;
}

int cfd_create(cfd_ctx** out, int device) {
  if (!out) return CFD_E_BADARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) return CFD_E_CUDA;
  if (device < 0) device = n - 1;  // CUDAcodes.cu:141-148 picks the last device
  if (device >= n) return CFD_E_BADARG;
  std::unique_ptr<cfd_ctx> c(new cfd_ctx());
  c->device = device;
  cfd_default_options(&c->opt);
  if (cudaSetDevice(device) != cudaSuccess) return CFD_E_CUDA;
  if (cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      c->num_sms < 1)
    return CFD_E_CUDA;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return CFD_E_CUDA;
  if (cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess) return CFD_E_CUDA;
  if (cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return CFD_E_CUDA;
  if (cudaMallocHost((void**)&c->h_small, 64 * sizeof(double)) != cudaSuccess) return CFD_E_CUDA;
  if (const char* e = std::getenv("CFD_FCG_GRAPH")) c->fcg_use_graph = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_FCG_PERSIST")) c->fcg_persist = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_COARSE_HOST")) c->coarse_on_host = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_PDL")) c->pdl = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_FCG_UPDATE_BLOCKS")) c->upd_grid = std::max(0, std::atoi(e));
  if (const char* e = std::getenv("CFD_HOST_PATTERNS")) c->host_patterns = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_L2_PERSIST")) c->l2_persist = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_COARSE_SPACING")) c->coarse_spacing = std::atof(e);
  if (const char* e = std::getenv("CFD_FCG_SPLIT")) c->fcg_split = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_CONVECT_TC")) c->convect_tc = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_FCG_ANCHOR")) c->fcg_anchor = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_SPLIT_SPMV_PER_SM")) c->split_spmv_per_sm = std::atoi(e) == 1 ? 1 : 2;
  *out = c.release();
  return CFD_OK;
}

void cfd_destroy(cfd_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream2) cudaStreamSynchronize(c->stream2);
  if (c->h_small) cudaFreeHost(c->h_small);
  if (c->l2_window) {
    // release the persisting L2 lines and the set-aside this context took
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.num_bytes = 0;
    if (c->stream) cudaStreamSetAttribute(c->stream, cudaStreamAttributeAccessPolicyWindow, &v);
    if (--g_l2_users == 0) {
      cudaCtxResetPersistingL2Cache();
      cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    }
  }
  cudaStream_t s = c->stream, s2 = c->stream2;
  cudaEvent_t e1 = c->ev_fork, e2 = c->ev_join;
  delete c;
  if (e1) cudaEventDestroy(e1);
  if (e2) cudaEventDestroy(e2);
  if (s2) cudaStreamDestroy(s2);
  if (s) cudaStreamDestroy(s);
}

const char* cfd_last_error(const cfd_ctx* c) { return c ? c->err.c_str() : "null context"; }

int cfd_set_options(cfd_ctx* c, const cfd_options* o) {
  if (!c || !o) return CFD_E_BADARG;
  NEED(o->precision == CFD_FP64 || o->precision == CFD_MIXED, "precision must be CFD_FP64 or CFD_MIXED");
  NEED(o->precond == CFD_PC_JACOBI || o->precond == CFD_PC_LEARNED || o->precond == CFD_PC_TWOLEVEL,
       "unknown preconditioner");
  NEED(o->cg_rtol > 0 && o->cg_rtol < 1, "cg_rtol must be in (0, 1)");
  NEED(o->cg_maxit > 0, "cg_maxit must be > 0");
  NEED(o->ngp_override == 0 || o->ngp_override == 1 || o->ngp_override == 8 || o->ngp_override == 27,
       "ngp_override must be 0, 1, 8 or 27");
  NEED(!c->loaded || o->precision == c->opt.precision, "precision must be set before cfd_load_inp");
  NEED(!c->loaded || o->ngp_override == c->opt.ngp_override, "ngp_override must be set before cfd_load_inp");
  c->opt = *o;
  if (c->opt.inner_rtol <= 0 || c->opt.inner_rtol >= 1) c->opt.inner_rtol = 1e-4;
  if (c->opt.max_outer <= 0) c->opt.max_outer = 12;
  if (c->opt.fcg_m <= 0) c->opt.fcg_m = 4;
  NEED(c->opt.fcg_m <= kFcgMaxM, "fcg_m must be in 1..8");
  NEED(c->opt.fcg_net_iters >= 0, "fcg_net_iters must be >= 0");
  return CFD_OK;
}

int cfd_load_inp(cfd_ctx* c, const char* path) {
  if (!c || !path) return CFD_E_BADARG;
  int rc = set_device(c);
  if (rc) return rc;
  c->P = HostProblem();
  rc = read_inp(path, c->P, c->err);
  if (rc) return rc;
  rc = preprocess(c->P, c->err, false);
  if (rc) return rc;
  return upload_problem(c);
}

int cfd_load_mesh(cfd_ctx* c, const cfd_problem_info* info, const double* coords, const int* conn, int nBC,
                  const double* bcvals, int nVelFaces, const int* velfaces, const double* monitor) {
  if (!c || !info || !coords || !conn || (nBC > 0 && !bcvals) || (nVelFaces > 0 && !velfaces) || !monitor)
    return CFD_E_BADARG;
  int rc = set_device(c);
  if (rc) return rc;
  HostProblem& P = c->P;
  P = HostProblem();
  P.NE = info->NE; P.NCN = info->NCN; P.NGP = info->NGP; P.maxIter = info->maxIter;
  P.dt = info->dt; P.t_ini = info->t_ini; P.t_final = info->t_final; P.tolerance = info->tolerance;
  P.convergence = info->convergence; P.density = info->density; P.viscosity = info->viscosity;
  P.zeroP = info->zeroPressureNode;
  NEED(P.NE > 0 && P.NCN > 0 && P.dt > 0 && P.maxIter > 0, "bad problem sizes");
  NEED(P.NGP == 1 || P.NGP == 8 || P.NGP == 27, "NGP must be 1, 8 or 27");
  // negative: no pin (the reference pins only p > 0); beyond the corner
  // nodes the pin would silently not apply and leave Z singular
  NEED(P.zeroP < P.NCN, "zero-pressure node out of range");
  P.NNp = P.NCN;
  P.coord.assign(coords, coords + 3 * (size_t)P.NCN);
  P.ltog.assign((size_t)P.NE * 27, -1);
  for (int e = 0; e < P.NE; e++)
    for (int i = 0; i < 8; i++) {
      int v = conn[(size_t)e * 8 + i];
      NEED(v >= 0 && v < P.NCN, "connectivity out of range");
      P.ltog[(size_t)e * 27 + i] = v;
    }
  P.nBC = nBC;
  P.bcstr.assign(bcvals, bcvals + 3 * (size_t)nBC);
  P.velfaces.assign(velfaces, velfaces + 3 * (size_t)nVelFaces);
  for (int i = 0; i < nVelFaces; i++) {
    NEED(velfaces[3 * i] >= 0 && velfaces[3 * i] < P.NE && velfaces[3 * i + 1] >= 0 && velfaces[3 * i + 1] < 6 &&
             velfaces[3 * i + 2] >= 0 && velfaces[3 * i + 2] < nBC,
         "velocity face out of range");
  }
  for (int d = 0; d < 3; d++) P.mon[d] = monitor[d];
  rc = preprocess(P, c->err, false);
  if (rc) return rc;
  return upload_problem(c);
}

int cfd_info(const cfd_ctx* c, cfd_problem_info* i) {
  if (!c || !i || !c->loaded) return CFD_E_BADARG;
  const HostProblem& P = c->P;
  std::memset(i, 0, sizeof(*i));
  i->NE = P.NE; i->NCN = P.NCN; i->NN = P.NN; i->NNp = P.NNp; i->NGP = P.NGP; i->maxIter = P.maxIter;
  i->nnzK = P.nnzK; i->nnzG = P.nnzG; i->nnzZ = P.nnzZ;
  i->nBCnodes = (int)P.bcnode.size(); i->monPoint = P.monPoint; i->zeroPressureNode = P.zeroP;
  i->dt = P.dt; i->t_ini = P.t_ini; i->t_final = P.t_final; i->tolerance = P.tolerance;
  i->convergence = P.convergence; i->density = P.density; i->viscosity = P.viscosity;
  i->timeN = c->timeN; i->timeT = c->timeT;
  return CFD_OK;
}

int cfd_step0(cfd_ctx* c) {
  if (!c) return CFD_E_BADARG;
  NEED(c->loaded, "cfd_step0 before cfd_load_inp");
  int rc = set_device(c);
  if (rc) return rc;
  HostProblem& P = c->P;
  cudaStream_t s = c->stream;
  for (auto* b : {&c->kval, &c->g1, &c->g2, &c->g3, &c->msum}) CU(cudaMemsetAsync(b->p, 0, b->bytes(), s));
  AsmArgs a{};
  a.NE = P.NE; a.ngp = P.NGP; a.ltog = c->ltog.p; a.coord = c->coord.p; a.basis = c->basis.p;
  a.viscosity = P.viscosity; a.inv_density = 1.0 / P.density;
  a.k_rp = c->k_rp.p; a.k_col = c->k_col.p; a.kval = c->kval.p;
  a.g_rp = c->g_rp.p; a.g_col = c->g_col.p; a.g1 = c->g1.p; a.g2 = c->g2.p; a.g3 = c->g3.p;
  a.msum = c->msum.p;
  if (c->opt.deterministic) {
    NEED(!c->color_off.empty(), "deterministic mode: the mesh needs more than 64 element colours");
    a.elist = c->elist.p;
    a.plain = 1;
    for (size_t k = 0; k + 1 < c->color_off.size(); k++) {
      a.e_begin = c->color_off[k];
      a.e_end = c->color_off[k + 1];
      CU(launch_assemble(a, c->num_sms, s));
    }
  } else {
    a.e_begin = 0;
    a.e_end = P.NE;
    CU(launch_assemble(a, c->num_sms, s));
  }
  CU(launch_fill_gt(P.nnzG, c->gt_pos.p, c->g1.p, c->g2.p, c->g3.p, c->gt1.p, c->gt2.p,
                    c->gt3.p, s));
  CU(launch_md_finalize(P.NN, c->msum.p, c->bcmask.p, c->minv_orig.p, c->minv_free.p, s));
  ZArgs z{};
  z.NNp = P.NNp; z.maxrow = std::max(1, P.maxZrow); z.zeroP = P.zeroP;
  z.z_rp = c->z_rp.p; z.z_col = c->z_col.p; z.zval = c->zval.p; z.zdiag = c->zdiag.p;
  z.gt_rp = c->gt_rp.p; z.gt_col = c->gt_col.p; z.gt1 = c->gt1.p; z.gt2 = c->gt2.p; z.gt3 = c->gt3.p;
  z.g_rp = c->g_rp.p; z.g_col = c->g_col.p; z.g1 = c->g1.p; z.g2 = c->g2.p; z.g3 = c->g3.p;
  z.minv_orig = c->minv_orig.p;
  CU(launch_build_z(z, s));
  CU(launch_recip(P.NNp, c->zdiag.p, c->zdinv.p, mixed(c) ? c->zdinv32.p : nullptr, s));
  // SELL-32 copies of the assembled operators (FP64, and FP32 in CFD_MIXED)
  CU(launch_csr_to_sell<double>(P.NN, c->k_rp.p, c->kval.p, c->ks_off.p, c->ks_val.p, s));
  CU(launch_csr_to_sell<double>(P.NN, c->g_rp.p, c->g1.p, c->gs_off.p, c->gs1.p, s));
  CU(launch_csr_to_sell<double>(P.NN, c->g_rp.p, c->g2.p, c->gs_off.p, c->gs2.p, s));
  CU(launch_csr_to_sell<double>(P.NN, c->g_rp.p, c->g3.p, c->gs_off.p, c->gs3.p, s));
  CU(launch_csr_to_sell<double>(P.NNp, c->gt_rp.p, c->gt1.p, c->gts_off.p, c->gts1.p, s));
  CU(launch_csr_to_sell<double>(P.NNp, c->gt_rp.p, c->gt2.p, c->gts_off.p, c->gts2.p, s));
  CU(launch_csr_to_sell<double>(P.NNp, c->gt_rp.p, c->gt3.p, c->gts_off.p, c->gts3.p, s));
  CU(launch_csr_to_sell<double>(P.NNp, c->z_rp.p, c->zval.p, c->zs_off.p, c->zs_val.p, s));
  if (mixed(c)) {
    CU(launch_csr_to_sell<float>(P.NN, c->k_rp.p, c->kval.p, c->ks_off.p, c->ks_val32.p, s));
    CU(launch_csr_to_sell<float>(P.NN, c->g_rp.p, c->g1.p, c->gs_off.p, c->gs1_32.p, s));
    CU(launch_csr_to_sell<float>(P.NN, c->g_rp.p, c->g2.p, c->gs_off.p, c->gs2_32.p, s));
    CU(launch_csr_to_sell<float>(P.NN, c->g_rp.p, c->g3.p, c->gs_off.p, c->gs3_32.p, s));
    CU(launch_csr_to_sell<float>(P.NNp, c->gt_rp.p, c->gt1.p, c->gts_off.p, c->gts1_32.p, s));
    CU(launch_csr_to_sell<float>(P.NNp, c->gt_rp.p, c->gt2.p, c->gts_off.p, c->gts2_32.p, s));
    CU(launch_csr_to_sell<float>(P.NNp, c->gt_rp.p, c->gt3.p, c->gts_off.p, c->gts3_32.p, s));
    CU(launch_csr_to_sell<float>(P.NNp, c->z_rp.p, c->zval.p, c->zs_off.p, c->zs_val32.p, s));
  }
  CU(cudaStreamSynchronize(s));
  c->assembled = true;
  c->coarse_ready = false;  // Z changed
  return CFD_OK;
}

int cfd_begin_step(cfd_ctx* c) {
  if (!c) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_begin_step before cfd_step0");
  cudaStream_t s = c->stream;
  const size_t NN = c->P.NN, NNp = c->P.NNp;
  c->timeN = c->timeN + 1;
  c->timeT = c->timeT + c->P.dt;
  CU(cudaMemcpyAsync(c->unphalf_prev, c->un, NN * sizeof(double4), cudaMemcpyDeviceToDevice, s));
  CU(cudaMemcpyAsync(c->pnp1_prev, c->pn, NNp * sizeof(double), cudaMemcpyDeviceToDevice, s));
  CU(cudaMemsetAsync(c->acc_prev, 0, NN * sizeof(double4), s));
  c->rotated = false;
  if (mixed(c)) {  // the gathered FP32 copies of the same vectors
    KL(CFD_K_OTHER, launch_vec4_to_f32((int)NN, c->un, c->un32, c->uphp32, s));
    CU(cudaMemsetAsync(c->accp32, 0, NN * sizeof(float4), s));
  }
  return CFD_OK;
}

int cfd_convect(cfd_ctx* c) {
  if (!c) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_convect before cfd_step0");
  cudaStream_t s = c->stream;
  if (mixed(c))
    CU(cudaMemsetAsync(c->r1c32, 0, c->P.NN * sizeof(float4), s));
  else
    CU(cudaMemsetAsync(c->r1conv, 0, c->P.NN * sizeof(double4), s));
  NEED(!c->opt.deterministic || !c->color_off.empty(),
       "deterministic mode: the mesh needs more than 64 element colours");
  auto run = [&](auto a, auto launch) -> int {
    if (c->opt.deterministic) {  // one colour per launch, plain adds
      a.elist = c->elist.p;
      a.plain = 1;
      for (size_t k = 0; k + 1 < c->color_off.size(); k++) {
        a.e_begin = c->color_off[k];
        a.e_end = c->color_off[k + 1];
        KL(CFD_K_CONVECT, launch(a));
      }
    } else {
      a.e_begin = 0;
      a.e_end = c->P.NE;
      KL(CFD_K_CONVECT, launch(a));
    }
    return CFD_OK;
  };
  if (mixed(c)) {
    ConvArgs<float> a{c->P.NE, c->P.NGP, c->ltog.p, c->coord.p, c->basis.p, c->un32, c->uphp32, c->r1conv};
    a.r1f = c->r1c32;
    if (c->convect_tc && !c->opt.deterministic) {
      a.e_begin = 0;
      a.e_end = c->P.NE;
      if (convect_tc_supported(a)) {
        if (!c->conv_err.p) {
          CU(c->conv_err.alloc(1));
          CU(cudaMemsetAsync(c->conv_err.p, 0, sizeof(int), s));
        }
        c->convect_tc_ran = true;
        KL(CFD_K_CONVECT, launch_convect_tc(a, c->conv_err.p, c->num_sms, s));
        return CFD_OK;
      }
    }
    return run(a, [&](const ConvArgs<float>& x) { return launch_convect<float>(x, c->num_sms, s); });
  }
  ConvArgs<double> a{c->P.NE, c->P.NGP, c->ltog.p, c->coord.p, c->basis.p, c->un, c->unphalf_prev, c->r1conv};
  return run(a, [&](const ConvArgs<double>& x) { return launch_convect<double>(x, c->num_sms, s); });
}

int cfd_step1(cfd_ctx* c, int iter) {
  if (!c) return CFD_E_BADARG;
  NEED(c->assembled && iter >= 1, "cfd_step1: bad state or iter");
  cudaStream_t s = c->stream;
  auto fill = [&](auto& a) {
    a.NN = c->P.NN; a.iter = iter; a.dt = c->P.dt;
    a.k_off = c->ks_off.p; a.k_col = c->ks_col.p; a.g_off = c->gs_off.p; a.g_col = c->gs_col.p;
    a.un = c->un; a.r1conv = c->r1conv; a.kacc = c->kacc;
    a.pn = c->pn; a.minv_free = c->minv_free.p; a.minv_orig = c->minv_orig.p;
    a.unphalf = c->unphalf; a.d = c->dvec; a.r1out = c->r_debug ? c->r1dbg : nullptr;
  };
  if (mixed(c)) {
    Step1Args<float> a{};
    fill(a);
    a.uprev = c->uphp32; a.unphalf_g = c->uph32; a.d_g = c->d32;
    a.r1conv32 = c->r1c32;
    a.kval = c->ks_val32.p; a.g1 = c->gs1_32.p; a.g2 = c->gs2_32.p; a.g3 = c->gs3_32.p;
    KL(CFD_K_STEP1, launch_step1<float>(a, c->num_sms, s));
  } else {
    Step1Args<double> a{};
    fill(a);
    a.uprev = c->unphalf_prev;
    a.kval = c->ks_val.p; a.g1 = c->gs1.p; a.g2 = c->gs2.p; a.g3 = c->gs3.p;
    KL(CFD_K_STEP1, launch_step1<double>(a, c->num_sms, s));
  }
  return CFD_OK;
}

int cfd_step2(cfd_ctx* c, int iter, cfd_solve_stats* st) {
  if (!c) return CFD_E_BADARG;
  NEED(c->assembled && iter >= 1, "cfd_step2: bad state or iter");
  cudaStream_t s = c->stream;
  const int pin = c->P.zeroP;
  if (mixed(c)) {
    GtArgs<float> a{c->P.NNp, pin, c->gts_off.p, c->gts_col.p, c->gts1_32.p, c->gts2_32.p, c->gts3_32.p, c->d32, c->r2};
    KL(CFD_K_GT, launch_gt<float>(a, c->num_sms, s));
  } else {
    GtArgs<double> a{c->P.NNp, pin, c->gts_off.p, c->gts_col.p, c->gts1.p, c->gts2.p, c->gts3.p, c->dvec, c->r2};
    KL(CFD_K_GT, launch_gt<double>(a, c->num_sms, s));
  }
  int rc = pressure_solve(c, c->r2, c->pdot, c->opt.cg_warm, st);
  if (rc) return rc;
  KL(CFD_K_PUPDATE, launch_pressure_update(c->P.NNp, c->P.dt, c->pn, c->pdot, c->pnp1_prev, c->pnp1, c->ppart.p, c->npb, s));
  return CFD_OK;
}

int cfd_step3(cfd_ctx* c, int iter) {
  if (!c) return CFD_E_BADARG;
  NEED(c->assembled && iter >= 1, "cfd_step3: bad state or iter");
  cudaStream_t s = c->stream;
  auto fill = [&](auto& a) {
    a.NN = c->P.NN; a.iter = iter; a.dt = c->P.dt;
    a.g_off = c->gs_off.p; a.g_col = c->gs_col.p; a.pdot = c->pdot; a.kacc = c->kacc; a.unphalf = c->unphalf;
    a.un = c->un; a.unp1_prev = c->unp1_prev; a.minv_free = c->minv_free.p; a.acc = c->acc; a.unp1 = c->unp1;
    a.r3out = c->r_debug ? c->r3dbg : nullptr; a.part = c->upart.p; a.nblocks = c->nub;
  };
  if (mixed(c)) {
    Step3Args<float> a{};
    fill(a);
    a.acc_g = c->acc32;
    a.g1 = c->gs1_32.p; a.g2 = c->gs2_32.p; a.g3 = c->gs3_32.p;
    KL(CFD_K_STEP3, launch_step3<float>(a, s));
  } else {
    Step3Args<double> a{};
    fill(a);
    a.g1 = c->gs1.p; a.g2 = c->gs2.p; a.g3 = c->gs3.p;
    KL(CFD_K_STEP3, launch_step3<double>(a, s));
  }
  c->rotated = false;
  return CFD_OK;
}

int cfd_check_iter(cfd_ctx* c, double tol, int* converged, double* norms) {
  if (!c || !converged) return CFD_E_BADARG;
  int rc = reduce_norms(c);
  if (rc) return rc;
  const double* v = c->last_norms;
  double n1 = std::sqrt(v[1]) / std::sqrt(v[0]);
  double n2 = std::sqrt(v[3]) / std::sqrt(v[2]);
  *converged = (n1 < tol && n2 < tol) ? 1 : 0;
  if (norms) {
    norms[0] = n1;
    norms[1] = n2;
  }
  return CFD_OK;
}

// The reference copies (UnpHalf_prev = UnpHalf, Unp1_prev = Unp1, ...,
// BCH.cpp:2964-2984), so the current vectors keep their values; here the
// buffers swap, and the current ones are rewritten by the next stages.
int cfd_rotate(cfd_ctx* c) {
  if (!c) return CFD_E_BADARG;
  c->rotated = true;
  std::swap(c->unphalf_prev, c->unphalf);
  std::swap(c->unp1_prev, c->unp1);
  std::swap(c->acc_prev, c->acc);
  std::swap(c->pnp1_prev, c->pnp1);
  std::swap(c->uphp32, c->uph32);
  std::swap(c->accp32, c->acc32);
  return CFD_OK;
}

int cfd_k_times_acc(cfd_ctx* c) {
  if (!c) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_k_times_acc before cfd_step0");
  cudaStream_t s = c->stream;
  if (mixed(c)) {
    SpmvK3Args<float> a{c->P.NN, c->ks_off.p, c->ks_col.p, c->ks_val32.p, c->accp32, c->kacc};
    KL(CFD_K_SPMV_K3, launch_spmv_k3<float>(a, c->num_sms, s));
  } else {
    SpmvK3Args<double> a{c->P.NN, c->ks_off.p, c->ks_col.p, c->ks_val.p, c->acc_prev, c->kacc};
    KL(CFD_K_SPMV_K3, launch_spmv_k3<double>(a, c->num_sms, s));
  }
  return CFD_OK;
}

int cfd_check_steady(cfd_ctx* c, double crit, double* maxAcc, int* steady) {
  if (!c) return CFD_E_BADARG;
  int rc = reduce_norms(c);
  if (rc) return rc;
  c->maxAcc = c->last_norms[4];
  if (maxAcc) *maxAcc = c->maxAcc;
  if (steady) *steady = (c->maxAcc > crit) ? 0 : 1;
  return CFD_OK;
}

// Un <- Unp1, Pn <- Pnp1 (BCH.cpp:3080-3081).  When the sub-iteration loop
// ran out (maxIter iterations without convergence), the last iteration was
// rotated: its Unp1 and Pnp1 are in the _prev buffers.  Unp1_prev must keep
// that Unp1 too (the next step's first convergence test compares against
// it, BCH.cpp:2874 being commented out), so the velocity is copied.
int cfd_end_step(cfd_ctx* c) {
  if (!c) return CFD_E_BADARG;
  if (c->rotated) {
    CU(cudaMemcpyAsync(c->un, c->unp1_prev, c->P.NN * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    std::swap(c->pn, c->pnp1_prev);
  } else {
    std::swap(c->un, c->unp1);
    std::swap(c->pn, c->pnp1);
  }
  c->rotated = false;
  return CFD_OK;
}

int cfd_run(cfd_ctx* c, int nsteps, cfd_run_stats* st) {
  if (!c) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_run before cfd_step0");
  cfd_run_stats r{};
  int rc = set_device(c);
  if (rc) return rc;
  const HostProblem& P = c->P;
  while (nsteps < 0 ? (c->timeT < P.t_final) : (r.steps < nsteps)) {
    if ((rc = cfd_begin_step(c))) return rc;
    int iter;
    for (iter = 1; iter <= P.maxIter; iter++) {
      cfd_solve_stats ss{};
      if ((rc = cfd_convect(c))) return rc;
      if ((rc = cfd_step1(c, iter))) return rc;
      if ((rc = cfd_step2(c, iter, &ss))) return rc;
      if ((rc = cfd_step3(c, iter))) return rc;
      r.cg_iters += ss.iterations;
      r.fallbacks += ss.fallback;
      r.subiters++;
      int conv = 0;
      if ((rc = cfd_check_iter(c, P.tolerance, &conv, nullptr))) return rc;
      if (conv) break;
      cfd_rotate(c);
      if ((rc = cfd_k_times_acc(c))) return rc;
    }
    r.last_iter = iter;
    int steady = 0;
    c->maxAcc = c->last_norms[4];
    steady = (c->maxAcc > P.convergence) ? 0 : 1;
    cfd_end_step(c);
    r.steps++;
    r.maxAcc = c->maxAcc;
    if (steady) {
      r.steady = 1;
      break;
    }
  }
  if (st) *st = r;
  return CFD_OK;
}

int cfd_get_monitor(cfd_ctx* c, int node, double* out) {
  if (!c || !out || !c->loaded) return CFD_E_BADARG;
  if (node < 0) node = c->P.monPoint;
  NEED(node < c->P.NN, "monitor node out of range");
  cudaStream_t s = c->stream;
  CU(cudaMemcpyAsync(c->h_small, c->un + node, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (node < c->P.NNp)
    CU(cudaMemcpyAsync(c->h_small + 3, c->pn + node, sizeof(double), cudaMemcpyDeviceToHost, s));
  else
    c->h_small[3] = 0.0;
  CU(cudaStreamSynchronize(s));
  for (int i = 0; i < 4; i++) out[i] = c->h_small[i];
  return CFD_OK;
}

int cfd_download_state(cfd_ctx* c, double* U, double* Pv) {
  if (!c || !c->loaded) return CFD_E_BADARG;
  cudaStream_t s = c->stream;
  if (U) {
    CU(launch_vec4_to_blocks(c->P.NN, c->un, c->blk.p, s));
    CU(cudaMemcpyAsync(U, c->blk.p, 3 * (size_t)c->P.NN * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  if (Pv) CU(cudaMemcpyAsync(Pv, c->pn, (size_t)c->P.NNp * sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  return CFD_OK;
}

int cfd_upload_state(cfd_ctx* c, const double* U, const double* Pv) {
  if (!c || !c->loaded) return CFD_E_BADARG;
  cudaStream_t s = c->stream;
  if (U) {
    CU(cudaMemcpyAsync(c->blk.p, U, 3 * (size_t)c->P.NN * sizeof(double), cudaMemcpyHostToDevice, s));
    CU(launch_blocks_to_vec4(c->P.NN, c->blk.p, c->un, s));
  }
  if (Pv) CU(cudaMemcpyAsync(c->pn, Pv, (size_t)c->P.NNp * sizeof(double), cudaMemcpyHostToDevice, s));
  CU(cudaStreamSynchronize(s));
  return CFD_OK;
}

int cfd_download_vector(cfd_ctx* c, int which, double* out) {
  if (!c || !out || !c->loaded) return CFD_E_BADARG;
  cudaStream_t s = c->stream;
  const size_t NN = c->P.NN, NNp = c->P.NNp;
  const double4* v4 = nullptr;
  const double* p1 = nullptr;
  switch (which) {
    case CFD_V_UN: v4 = c->un; break;
    case CFD_V_UNP1: v4 = c->unp1; break;
    case CFD_V_UNP1_PREV: v4 = c->unp1_prev; break;
    case CFD_V_UNPHALF: v4 = c->unphalf; break;
    case CFD_V_UNPHALF_PREV: v4 = c->unphalf_prev; break;
    case CFD_V_ACC: v4 = c->acc; break;
    case CFD_V_ACC_PREV: v4 = c->acc_prev; break;
    case CFD_V_KACC_PREV: v4 = c->kacc; break;
    case CFD_V_R1: v4 = c->r1dbg; break;
    case CFD_V_R3: v4 = c->r3dbg; break;
    case CFD_V_PN: p1 = c->pn; break;
    case CFD_V_PNP1: p1 = c->pnp1; break;
    case CFD_V_PNP1_PREV: p1 = c->pnp1_prev; break;
    case CFD_V_PDOT: p1 = c->pdot; break;
    case CFD_V_R2: p1 = c->r2; break;
    case CFD_V_MDINV:
    case CFD_V_MDORIGINV: {
      NEED(c->assembled, "mass matrix not assembled");
      std::vector<double> m(NN);
      std::vector<unsigned char> bc(NN);
      CU(cudaMemcpyAsync(m.data(), c->minv_orig.p, NN * sizeof(double), cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
      for (int i : c->P.bcnode) bc[i] = 1;
      for (size_t i = 0; i < NN; i++) {
        double v = (which == CFD_V_MDINV && bc[i]) ? 1.0 : m[i];
        out[i] = out[NN + i] = out[2 * NN + i] = v;
      }
      return CFD_OK;
    }
    case CFD_V_DIV: {
      NEED(c->assembled, "operators not assembled");
      GtArgs<double> a{(int)NNp, 0, c->gts_off.p, c->gts_col.p, c->gts1.p, c->gts2.p, c->gts3.p, c->unp1, c->ir_r.p};
      CU(launch_gt<double>(a, c->num_sms, s));
      p1 = c->ir_r.p;
      break;
    }
    default:
      return fail(c, CFD_E_BADARG, "unknown vector id %d", which);
  }
  if (v4) {
    CU(launch_vec4_to_blocks((int)NN, v4, c->blk.p, s));
    CU(cudaMemcpyAsync(out, c->blk.p, 3 * NN * sizeof(double), cudaMemcpyDeviceToHost, s));
  } else {
    CU(cudaMemcpyAsync(out, p1, NNp * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CU(cudaStreamSynchronize(s));
  return CFD_OK;
}

int cfd_download_matrix(cfd_ctx* c, int which, long long* nnz, int* rowptr, int* col, double* val) {
  if (!c || !c->loaded) return CFD_E_BADARG;
  if (col) {
    int rc = ensure_host_columns(c);
    if (rc) return rc;
  }
  const HostProblem& P = c->P;
  const std::vector<int>* rp = nullptr;
  const std::vector<int>* cl = nullptr;
  const double* v[3] = {nullptr, nullptr, nullptr};
  switch (which) {
    case CFD_M_K: rp = &P.k_rp; cl = &P.k_col; v[0] = c->kval.p; break;
    case CFD_M_G: rp = &P.g_rp; cl = &P.g_col; v[0] = c->g1.p; v[1] = c->g2.p; v[2] = c->g3.p; break;
    case CFD_M_GT: rp = &P.gt_rp; cl = &P.gt_col; v[0] = c->gt1.p; v[1] = c->gt2.p; v[2] = c->gt3.p; break;
    case CFD_M_Z: rp = &P.z_rp; cl = &P.z_col; v[0] = c->zval.p; break;
    default: return fail(c, CFD_E_BADARG, "unknown matrix id %d", which);
  }
  const size_t n = which == CFD_M_K ? (size_t)P.nnzK : which == CFD_M_Z ? (size_t)P.nnzZ : (size_t)P.nnzG;
  if (nnz) *nnz = (long long)n;
  if (rowptr) std::copy(rp->begin(), rp->end(), rowptr);
  if (col) std::copy(cl->begin(), cl->end(), col);
  if (val) {
    NEED(c->assembled, "operators not assembled");
    cudaStream_t s = c->stream;
    if (!v[1]) {
      CU(cudaMemcpyAsync(val, v[0], n * sizeof(double), cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
    } else {
      std::vector<double> t(n);
      for (int d = 0; d < 3; d++) {
        CU(cudaMemcpyAsync(t.data(), v[d], n * sizeof(double), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        for (size_t i = 0; i < n; i++) val[3 * i + d] = t[i];
      }
    }
  }
  return CFD_OK;
}

int cfd_pressure_solve(cfd_ctx* c, const double* rhs, double* x, cfd_solve_stats* st) {
  if (!c || !rhs || !x) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_pressure_solve before cfd_step0");
  cudaStream_t s = c->stream;
  const size_t NNp = c->P.NNp;
  // use r2 as the right-hand side slot and pdot as the solution slot
  CU(cudaMemcpyAsync(c->r2, rhs, NNp * sizeof(double), cudaMemcpyHostToDevice, s));
  if (c->opt.cg_warm) CU(cudaMemcpyAsync(c->pdot, x, NNp * sizeof(double), cudaMemcpyHostToDevice, s));
  int rc = pressure_solve(c, c->r2, c->pdot, c->opt.cg_warm, st);
  if (rc && rc != CFD_E_NOCONV) return rc;
  CU(cudaMemcpyAsync(x, c->pdot, NNp * sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  return rc;
}

int cfd_write_tecplot(cfd_ctx* c, const char* path, const char* title) {
  if (!c || !path || !c->loaded) return CFD_E_BADARG;
  std::vector<double> U(3 * (size_t)c->P.NN), Pv(c->P.NNp);
  int rc = cfd_download_state(c, U.data(), Pv.data());
  if (rc) return rc;
  rc = write_tecplot(c->P, U.data(), Pv.data(), path, title ? title : "");
  if (rc) return fail(c, rc, "cannot write %s", path);
  return CFD_OK;
}

int cfd_read_restart(cfd_ctx* c, const char* path) {
  if (!c || !path || !c->loaded) return CFD_E_BADARG;
  std::vector<double> U(3 * (size_t)c->P.NN, 0.0), Pv(c->P.NNp, 0.0);
  int rc = read_restart(c->P, path, U.data(), Pv.data());
  if (rc) return fail(c, rc, "cannot read restart file %s", path);
  return cfd_upload_state(c, U.data(), Pv.data());
}

int cfd_set_bc_values(cfd_ctx* c, int n, const int* nodes, const double* uvw) {
  if (!c || !c->loaded || n < 0 || (n > 0 && (!nodes || !uvw))) return CFD_E_BADARG;
  for (int i = 0; i < n; i++) NEED(nodes[i] >= 0 && nodes[i] < c->P.NN, "BC node out of range");
  DevBuf<int> dn;
  DevBuf<double> dv;
  cudaStream_t s = c->stream;
  CU(dn.alloc(n));
  CU(dv.alloc(3 * (size_t)n));
  CU(cudaMemcpyAsync(dn.p, nodes, n * sizeof(int), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(dv.p, uvw, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  CU(launch_apply_bc(n, dn.p, dv.p, c->un, s));
  CU(cudaStreamSynchronize(s));
  return CFD_OK;
}

void* cfd_stream(cfd_ctx* c) { return c ? (void*)c->stream : nullptr; }

long long cfd_launch_count(const cfd_ctx* c) { return c ? c->launches : -1; }

int cfd_profile(cfd_ctx* c, int on) {
  if (!c) return CFD_E_BADARG;
  cudaStream_t s = c->stream;
  CU(cudaStreamSynchronize(s));
  harvest(c);
  if (on) {
    std::memset(c->prof, 0, sizeof(c->prof));
    if (c->fcg2l_time.p) CU(cudaMemset(c->fcg2l_time.p, 0, c->fcg2l_time.bytes()));
  }
  c->prof_on = on != 0;
  return CFD_OK;
}

int cfd_profile_fcg2l(cfd_ctx* c, double* out10) {
  if (!c || !out10) return CFD_E_BADARG;
  CU(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 10; k++) out10[k] = 0.0;
  if (!c->fcg2l_time.p) return CFD_OK;
  std::vector<double> t(c->fcg2l_time.n);
  CU(cudaMemcpy(t.data(), c->fcg2l_time.p, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int k = 0; k < 7; k++) out10[k] = t[k] * 1e-6;
  const int G = (int)t.size() - 8;
  if (G > 0) {
    double mn = t[8], mx = t[8], sum = 0.0;
    for (int b = 0; b < G; b++) {
      mn = std::min(mn, t[8 + b]);
      mx = std::max(mx, t[8 + b]);
      sum += t[8 + b];
    }
    out10[7] = mn * 1e-6;
    out10[8] = sum / G * 1e-6;
    out10[9] = mx * 1e-6;
  }
  return CFD_OK;
}

int cfd_profile_read(cfd_ctx* c, double* out) {
  if (!c || !out) return CFD_E_BADARG;
  CU(cudaStreamSynchronize(c->stream));
  harvest(c);
  for (int k = 0; k < CFD_K_COUNT; k++)
    for (int j = 0; j < 3; j++) out[3 * k + j] = c->prof[k][j];
  return CFD_OK;
}

int cfd_spd_inverse(int device, const double* a, int n, double* inv) {
  if (!a || !inv || n < 1 || n > 16384) return CFD_E_BADARG;
  if (cudaSetDevice(device) != cudaSuccess) return CFD_E_CUDA;
  const int ld = spd_inverse_ld(n);
  DevBuf<double> dA, dW;
  DevBuf<int> dinfo;
  if (dA.alloc((size_t)ld * ld) != cudaSuccess || dW.alloc((size_t)ld * ld) != cudaSuccess ||
      dinfo.alloc(1) != cudaSuccess)
    return CFD_E_NOMEM;
  int info = 0;
  cudaError_t e = cudaMemcpy2D(dA.p, ld * sizeof(double), a, n * sizeof(double), n * sizeof(double), n,
                               cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = spd_inverse_device(dA.p, dW.p, n, ld, dinfo.p, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(&info, dinfo.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy2D(inv, n * sizeof(double), dA.p, ld * sizeof(double), n * sizeof(double), n,
                     cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return CFD_E_CUDA;
  return info == 0 ? CFD_OK : CFD_E_NONFINITE;
}

int cfd_coarse_matrix(int device, const int dims[3], const int* rowptr, const int* col, const double* val,
                      double spacing, int* cd, double* zc) {
  if (!dims || !rowptr || !col || !val || !cd) return CFD_E_BADARG;
  const long long n = (long long)dims[0] * dims[1] * dims[2];
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || n > (1LL << 30)) return CFD_E_BADARG;
  double h[3];
  coarse_lattice(dims, kCoarseMaxNodes, cd, h, spacing);
  if (!zc) return CFD_OK;
  if (cudaSetDevice(device) != cudaSuccess) return CFD_E_CUDA;
  const int np = (int)n, nc = cd[0] * cd[1] * cd[2];
  const long long nnz = rowptr[np];
  if (nnz < 0 || nnz > (1LL << 31) - 1) return CFD_E_BADARG;
  DevBuf<int> i0[3], rng[3], drp, dcol, wlo, bad;
  DevBuf<double> f[3], dval, w27, dzc;
  cudaError_t e = cudaSuccess;
  for (int a = 0; a < 3 && e == cudaSuccess; a++) {
    std::vector<int> hi0, hrng;
    std::vector<double> hf;
    hat_tables(dims[a], cd[a], h[a], hi0, hf, hrng);
    e = i0[a].alloc(dims[a]);
    if (e == cudaSuccess) e = f[a].alloc(dims[a]);
    if (e == cudaSuccess) e = rng[a].alloc(hrng.size());
    if (e == cudaSuccess) e = cudaMemcpy(i0[a].p, hi0.data(), dims[a] * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(f[a].p, hf.data(), dims[a] * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(rng[a].p, hrng.data(), hrng.size() * sizeof(int), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = drp.alloc(np + 1);
  if (e == cudaSuccess) e = dcol.alloc(std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = dval.alloc(std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = w27.alloc(27 * (size_t)np);
  if (e == cudaSuccess) e = wlo.alloc(np);
  if (e == cudaSuccess) e = bad.alloc(1);
  if (e == cudaSuccess) e = dzc.alloc((size_t)nc * nc);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? CFD_E_NOMEM : CFD_E_CUDA;
  e = cudaMemcpy(drp.p, rowptr, (np + 1) * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dcol.p, col, nnz * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dval.p, val, nnz * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(bad.p, 0, sizeof(int));
  GalerkinArgs g{};
  for (int a = 0; a < 3; a++) {
    g.fd[a] = dims[a];
    g.cd[a] = cd[a];
  }
  g.np = np;
  g.nc = nc;
  g.i0x = i0[0].p;
  g.i0y = i0[1].p;
  g.i0z = i0[2].p;
  g.fx = f[0].p;
  g.fy = f[1].p;
  g.fz = f[2].p;
  g.rx = rng[0].p;
  g.ry = rng[1].p;
  g.rz = rng[2].p;
  g.rp = drp.p;
  g.col = dcol.p;
  g.val = dval.p;
  g.w27 = w27.p;
  g.wlo = wlo.p;
  g.bad = bad.p;
  g.zc = dzc.p;
  g.ld = nc;
  if (e == cudaSuccess) e = launch_galerkin(g, nullptr);
  int hb = 1;
  if (e == cudaSuccess) e = cudaMemcpy(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && hb == 0) e = cudaMemcpy(zc, dzc.p, (size_t)nc * nc * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return CFD_E_CUDA;
  return hb == 0 ? CFD_OK : CFD_E_BADINPUT;
}

int cfd_selftest_wait_timeout(cfd_ctx* c, int timeout_ms) {
  if (!c || timeout_ms <= 0 || timeout_ms > 10000) return CFD_E_BADARG;
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t s = c->stream;
  DevBuf<int> flags;
  CU(flags.alloc(2));
  CU(cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), s));
  KL(CFD_K_OTHER, launch_wait_selftest(flags.p, flags.p + 1, (unsigned long long)timeout_ms * 1000000ULL, s));
  int h[2] = {0, 0};
  CU(cudaMemcpyAsync(h, flags.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (h[1]) return fail(c, CFD_E_TIMEOUT, "bounded wait gave up after %d ms (self-test)", timeout_ms);
  return CFD_OK;
}

int cfd_unet_create(cfd_unet** out, int device, unsigned long long seed) {
  if (!out) return CFD_E_BADARG;
  *out = nullptr;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return CFD_E_CUDA;
  std::unique_ptr<cfd_unet> u(new cfd_unet());
  if (u->net.init(seed)) return CFD_E_CUDA;
  *out = u.release();
  return CFD_OK;
}

void cfd_unet_destroy(cfd_unet* u) {
  if (!u) return;
  cudaSetDevice(u->net.device);
  cudaDeviceSynchronize();
  delete u;
}

const char* cfd_unet_last_error(const cfd_unet* u) { return u ? u->net.err.c_str() : "null network"; }

long long cfd_unet_param_count(void) { return unet_param_count(); }

int cfd_unet_get_params(cfd_unet* u, float* out, long long n) {
  if (!u || !out) return CFD_E_BADARG;
  cudaSetDevice(u->net.device);
  if (cudaStreamSynchronize(u->net.own_stream) != cudaSuccess) return CFD_E_CUDA;
  return u->net.get_params(out, n) ? CFD_E_BADARG : CFD_OK;
}

int cfd_unet_set_params(cfd_unet* u, const float* in, long long n) {
  if (!u || !in) return CFD_E_BADARG;
  cudaSetDevice(u->net.device);
  cudaDeviceSynchronize();
  return u->net.set_params(in, n) ? CFD_E_BADARG : CFD_OK;
}

int cfd_unet_save(cfd_unet* u, const char* path) {
  if (!u || !path) return CFD_E_BADARG;
  std::vector<float> h((size_t)u->net.nparam);
  int rc = cfd_unet_get_params(u, h.data(), u->net.nparam);
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    u->net.err = std::string("cannot write ") + path;
    return CFD_E_IO;
  }
  const long long n = u->net.nparam;
  bool ok = std::fwrite("CFDUNET1", 1, 8, f) == 8 && std::fwrite(&n, sizeof(n), 1, f) == 1 &&
            std::fwrite(h.data(), sizeof(float), h.size(), f) == h.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) u->net.err = std::string("short write to ") + path;
  return ok ? CFD_OK : CFD_E_IO;
}

int cfd_unet_read(cfd_unet* u, const char* path) {
  if (!u || !path) return CFD_E_BADARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    u->net.err = std::string("cannot open ") + path;
    return CFD_E_IO;
  }
  char tag[8] = {0};
  long long n = 0;
  std::vector<float> h;
  bool ok = std::fread(tag, 1, 8, f) == 8 && std::memcmp(tag, "CFDUNET1", 8) == 0 &&
            std::fread(&n, sizeof(n), 1, f) == 1 && n == u->net.nparam;
  if (ok) {
    h.resize((size_t)n);
    ok = std::fread(h.data(), sizeof(float), h.size(), f) == h.size();
  }
  std::fclose(f);
  if (!ok) {
    u->net.err = std::string("not a weight file of this network: ") + path;
    return CFD_E_BADINPUT;
  }
  return cfd_unet_set_params(u, h.data(), n);
}

namespace {

int unet_prepare(cfd_unet* u, const int* dims, bool train, long long* nv) {
  if (!dims) return CFD_E_BADARG;
  cudaSetDevice(u->net.device);
  if (u->net.set_grid(dims, train)) return CFD_E_BADARG;
  *nv = u->net.nvox[0];
  return CFD_OK;
}

// act[0] <- bf16(x) for sample x (host or device FP32)
int unet_load_input(cfd_unet* u, const float* x, long long nv, int on_device, float* dev_tmp) {
  cudaStream_t s = u->net.own_stream;
  const float* src = x;
  if (!on_device) {
    if (cudaMemcpyAsync(dev_tmp, x, nv * sizeof(float), cudaMemcpyHostToDevice, s)) return CFD_E_CUDA;
    src = dev_tmp;
  }
  u->net.launches++;
  return unet_input((int)nv, src, nullptr, nullptr, 1.0, u->net.act[0], nullptr, s) ? CFD_E_CUDA : CFD_OK;
}

}  // namespace

int cfd_unet_forward(cfd_unet* u, const int dims[3], const float* x, float* y, int on_device) {
  if (!u || !x || !y) return CFD_E_BADARG;
  long long nv = 0;
  int rc = unet_prepare(u, dims, false, &nv);
  if (rc) return rc;
  UnetNet& n = u->net;
  cudaStream_t s = n.own_stream;
  DevBuf<float> tmp;
  if (!on_device && tmp.alloc(2 * (size_t)nv)) return CFD_E_NOMEM;
  rc = unet_load_input(u, x, nv, on_device, tmp.p);
  if (rc) return rc;
  // the output stays in the network's FP32 buffer too (cfd_unet_tensor)
  if (n.forward(s, nullptr) != cudaSuccess) return CFD_E_CUDA;
  if (cudaMemcpyAsync(y, n.out, nv * sizeof(float), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                      s))
    return CFD_E_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? CFD_OK : CFD_E_CUDA;
}

namespace {

// forward + MSE + backward of one sample; gradients accumulate into G
int unet_sample(cfd_unet* u, const float* x, const float* t, long long nv, int on_device, float* tmp) {
  UnetNet& n = u->net;
  cudaStream_t s = n.own_stream;
  int rc = unet_load_input(u, x, nv, on_device, tmp);
  if (rc) return rc;
  const float* tg = t;
  if (!on_device) {
    if (cudaMemcpyAsync(tmp + nv, t, nv * sizeof(float), cudaMemcpyHostToDevice, s)) return CFD_E_CUDA;
    tg = tmp + nv;
  }
  if (n.forward(s, nullptr) != cudaSuccess) return CFD_E_CUDA;
  n.launches++;
  if (unet_loss(n.dims[0], n.out, tg, n.grad[kUnetTensors - 1], n.lossv, n.w_l2, n.w_h1, s) != cudaSuccess)
    return CFD_E_CUDA;
  return n.backward(s) == cudaSuccess ? CFD_OK : CFD_E_CUDA;
}

}  // namespace

int cfd_unet_gradient(cfd_unet* u, const int dims[3], const float* x, const float* t, int on_device, float* loss,
                      float* grad) {
  if (!u || !x || !t) return CFD_E_BADARG;
  long long nv = 0;
  int rc = unet_prepare(u, dims, true, &nv);
  if (rc) return rc;
  UnetNet& n = u->net;
  cudaStream_t s = n.own_stream;
  DevBuf<float> tmp;
  if (!on_device && tmp.alloc(2 * (size_t)nv)) return CFD_E_NOMEM;
  if (cudaMemsetAsync(n.G, 0, n.nparam * sizeof(float), s) || cudaMemsetAsync(n.lossv, 0, sizeof(float), s))
    return CFD_E_CUDA;
  rc = unet_sample(u, x, t, nv, on_device, tmp.p);
  if (rc) return rc;
  if (cudaMemcpyAsync(n.h_pinned, n.lossv, sizeof(float), cudaMemcpyDeviceToHost, s)) return CFD_E_CUDA;
  if (grad && cudaMemcpyAsync(grad, n.G, n.nparam * sizeof(float), cudaMemcpyDeviceToHost, s)) return CFD_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return CFD_E_CUDA;
  if (loss) *loss = n.h_pinned[0];
  return CFD_OK;
}

int cfd_unet_tensor(cfd_unet* u, int t, float* out, long long n) {
  if (!u || !out || t < 0 || t >= kUnetTensors) return CFD_E_BADARG;
  UnetNet& net = u->net;
  const long long need = net.nvox[kUnetTensor[t].level] * kUnetTensor[t].ch;
  if (n != need || need == 0) {
    net.err = "tensor size mismatch (or no forward pass yet)";
    return CFD_E_BADARG;
  }
  cudaSetDevice(net.device);
  if (cudaStreamSynchronize(net.own_stream) != cudaSuccess) return CFD_E_CUDA;
  if (t == kUnetTensors - 1)
    return cudaMemcpy(out, net.out, n * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? CFD_OK : CFD_E_CUDA;
  std::vector<uint16_t> h((size_t)n);
  if (cudaMemcpy(h.data(), net.act[t], n * sizeof(uint16_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    return CFD_E_CUDA;
  for (long long i = 0; i < n; i++) {
    const uint32_t b = (uint32_t)h[(size_t)i] << 16;
    std::memcpy(out + i, &b, sizeof(float));
  }
  return CFD_OK;
}

int cfd_unet_set_tensor_cores(cfd_unet* u, int on) {
  if (!u) return CFD_E_BADARG;
  u->net.tc_enabled = on != 0;
  return CFD_OK;
}

int cfd_unet_status(cfd_unet* u) {
  if (!u) return CFD_E_BADARG;
  cudaSetDevice(u->net.device);
  int h = 0;
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(&h, u->net.tc_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return CFD_E_CUDA;
  if (h) {
    u->net.err = "a bounded wait in a tensor-core convolution gave up";
    return CFD_E_TIMEOUT;
  }
  return CFD_OK;
}

int cfd_unet_set_loss(cfd_unet* u, float w_l2, float w_h1) {
  if (!u || !(w_l2 >= 0) || !(w_h1 >= 0) || w_l2 + w_h1 <= 0) return CFD_E_BADARG;
  u->net.w_l2 = w_l2;
  u->net.w_h1 = w_h1;
  return CFD_OK;
}

int cfd_unet_train_batch(cfd_unet* u, const int dims[3], int nb, const float* x, const float* t, int on_device,
                         float lr, float* loss) {
  if (!u || !x || !t || nb < 1 || !(lr > 0)) return CFD_E_BADARG;
  long long nv = 0;
  int rc = unet_prepare(u, dims, true, &nv);
  if (rc) return rc;
  UnetNet& n = u->net;
  cudaStream_t s = n.own_stream;
  DevBuf<float> tmp;
  if (!on_device && tmp.alloc(2 * (size_t)nv)) return CFD_E_NOMEM;
  if (cudaMemsetAsync(n.G, 0, n.nparam * sizeof(float), s) || cudaMemsetAsync(n.lossv, 0, sizeof(float), s))
    return CFD_E_CUDA;
  for (int i = 0; i < nb; i++) {
    rc = unet_sample(u, x + (size_t)i * nv, t + (size_t)i * nv, nv, on_device, tmp.p);
    if (rc) return rc;
  }
  if (n.adam(s, lr, 1.0f / nb) != cudaSuccess) return CFD_E_CUDA;
  if (cudaMemcpyAsync(n.h_pinned, n.lossv, sizeof(float), cudaMemcpyDeviceToHost, s)) return CFD_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return CFD_E_CUDA;
  if (loss) *loss = n.h_pinned[0] / nb;
  return CFD_OK;
}

int cfd_unet_attach(cfd_ctx* c, cfd_unet* u, const int dims[3], const int* p_of_vox) {
  if (!c) return CFD_E_BADARG;
  if (!u) {
    c->reset_fcg_graphs();
    c->unet = nullptr;
    c->unet_owned.reset();
    return CFD_OK;
  }
  NEED(c->assembled, "cfd_unet_attach before cfd_step0");
  NEED(dims, "cfd_unet_attach needs the grid dims");
  NEED(u->net.device == c->device, "network and context live on different devices");
  const long long nv = (long long)dims[0] * dims[1] * dims[2];
  NEED(nv == c->P.NNp, "grid dims do not multiply to the number of pressure nodes");
  if (u->net.set_grid(dims, false)) return fail(c, CFD_E_BADARG, "%s", u->net.err.c_str());
  const bool same = c->grid_set && dims[0] == c->udims[0] && dims[1] == c->udims[1] && dims[2] == c->udims[2] &&
                    (p_of_vox ? c->h_pmap.size() == (size_t)nv &&
                                    std::equal(c->h_pmap.begin(), c->h_pmap.end(), p_of_vox)
                              : c->h_pmap.empty());
  if (!same) {
    int rc = set_grid(c, dims, p_of_vox);
    if (rc) return rc;
  }
  c->reset_fcg_graphs();
  {
    std::vector<double> dg(nv);
    CU(cudaStreamSynchronize(c->stream));
    CU(cudaMemcpy(dg.data(), c->zdiag.p, nv * sizeof(double), cudaMemcpyDeviceToHost));
    std::nth_element(dg.begin(), dg.begin() + nv / 2, dg.end());
    c->unet_dscale = dg[nv / 2] > 0 ? dg[nv / 2] : 1.0;
  }
  if (c->unet_owned.get() != u) c->unet_owned.reset();
  c->unet = u;
  return CFD_OK;
}

int cfd_unet_load(cfd_ctx* c, const char* path, const int dims[3]) {
  if (!c || !path) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_unet_load before cfd_step0");
  int d[3];
  if (dims) {
    for (int a = 0; a < 3; a++) d[a] = dims[a];
  } else {
    int m = (int)std::llround(std::cbrt((double)c->P.NNp));
    NEED((long long)m * m * m == c->P.NNp, "pressure nodes do not form a cube: pass the grid dims");
    d[0] = d[1] = d[2] = m;
  }
  CU(cudaSetDevice(c->device));
  cfd_unet* u = nullptr;
  int rc = cfd_unet_create(&u, c->device, 0);
  if (rc) return fail(c, rc, "cannot create the network");
  std::unique_ptr<cfd_unet> own(u);
  rc = cfd_unet_read(u, path);
  if (rc) return fail(c, rc, "%s", u->net.err.c_str());
  c->unet_owned.reset();
  rc = cfd_unet_attach(c, u, d, nullptr);
  if (rc) return rc;
  c->unet_owned = std::move(own);
  return CFD_OK;
}

int cfd_pressure_residual(cfd_ctx* c, const double* rhs, const double* x, double* r, double* norm) {
  if (!c || !rhs || !x || !r) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_pressure_residual before cfd_step0");
  cudaStream_t s = c->stream;
  const size_t NNp = c->P.NNp;
  DevBuf<double> db, dx;
  CU(db.alloc(NNp));
  CU(dx.alloc(NNp));
  CU(cudaMemcpyAsync(db.p, rhs, NNp * sizeof(double), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(dx.p, x, NNp * sizeof(double), cudaMemcpyHostToDevice, s));
  double nr = 0;
  int rc = residual_norm(c, db.p, dx.p, &nr);
  if (rc) return rc;
  CU(cudaMemcpyAsync(r, c->ir_r.p, NNp * sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (norm) *norm = nr;
  return CFD_OK;
}

int cfd_set_pressure_grid(cfd_ctx* c, const int dims[3], const int* p_of_vox) {
  if (!c || !dims) return CFD_E_BADARG;
  NEED(c->loaded, "cfd_set_pressure_grid before cfd_load_inp");
  return set_grid(c, dims, p_of_vox);
}

int cfd_precond_apply(cfd_ctx* c, const double* r, double* z) {
  if (!c || !r || !z) return CFD_E_BADARG;
  NEED(c->assembled, "cfd_precond_apply before cfd_step0");
  cudaStream_t s = c->stream;
  const bool with_coarse = c->opt.precond == CFD_PC_TWOLEVEL || c->opt.precond == CFD_PC_LEARNED;
  if (with_coarse) {
    int rc = ensure_coarse(c);
    if (rc) return rc;
  }
  const size_t NNp = c->P.NNp;
  DevBuf<double> dr, dz;
  CU(dr.alloc(NNp));
  CU(dz.alloc(NNp));
  CU(cudaMemcpyAsync(dr.p, r, NNp * sizeof(double), cudaMemcpyHostToDevice, s));
  CoarseArgs<double> ca{};
  if (with_coarse) {
    ca = coarse_args<double>(c, true);
  } else {  // Jacobi: position-independent, no grid needed
    ca.fd[0] = (int)NNp;
    ca.fd[1] = ca.fd[2] = 1;
  }
  if (with_coarse) {
    CU(launch_coarse_restrict<double>(ca, dr.p, c->cs_c32.p, nullptr, s));
    CU(launch_coarse_solve<double>(ca, c->cs_c32.p, c->cs_e64.p, nullptr, s));
  }
  CU(launch_precond<double>(ca, (int)NNp, dr.p, c->zdinv.p, with_coarse ? c->cs_e64.p : nullptr, nullptr, nullptr,
                            1.0, dz.p, nullptr, s));
  c->launches += with_coarse ? 3 : 1;
  CU(cudaMemcpyAsync(z, dz.p, NNp * sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  return CFD_OK;
}

}  // extern "C"
