/*
 * cfdfs.h -- C ABI of the B200 fractional-step solver (libcfdfs.so).
 *
 * Drop-in replacement for the device seam of the reference solver: the eleven
 * C++ functions that fractionalStep/Cpp/blascoCodinaHuerta.cpp declares at
 * lines 365-377 and that fractionalStep/Cpp/CUDAcodes.cu defines, plus the
 * host preprocessing of blascoCodinaHuerta.cpp:528-2711 that feeds them.
 * Each entry point names the reference function it replaces.
 *
 * Conventions
 *   - Every call returns CFD_OK (0) or a negative CFD_E_* code; none blocks
 *     on user input or exits (the reference prints "ErrorNN" and waits on
 *     std::cin, e.g. CUDAcodes.cu:184-250).  cfd_last_error() gives text.
 *   - One context = one GPU, one CUDA stream, single-threaded use.
 *   - Host buffers belong to the caller; device buffers to the context.
 *   - Vectors crossing the ABI use the reference layout: velocity as three
 *     component blocks [u(0..NN-1) | v | w] (blascoCodinaHuerta.cpp:1348-1368),
 *     pressure on the NNp corner nodes.  Node numbers are the reference's
 *     (corner nodes first, then mid-edge, mid-face and centre nodes).
 */
#ifndef CFDFS_H
#define CFDFS_H

#ifdef __cplusplus
extern "C" {
#endif

#define CFDFS_ABI_VERSION 1

enum cfd_status {
  CFD_OK = 0,
  CFD_E_CUDA = -1,      /* CUDA runtime error or no usable device */
  CFD_E_NOCONV = -2,    /* Krylov solve hit its iteration limit */
  CFD_E_NONFINITE = -3, /* NaN/Inf in a residual or norm */
  CFD_E_TIMEOUT = -4,   /* a bounded device-side wait gave up */
  CFD_E_BADARG = -5,    /* invalid argument or call order */
  CFD_E_BADINPUT = -6,  /* malformed .inp deck */
  CFD_E_IO = -7,        /* file could not be opened / written */
  CFD_E_NOMEM = -8      /* device allocation failed */
};

enum cfd_precision {
  CFD_FP64 = 0,  /* all operators, vectors and Krylov work in FP64 */
  CFD_MIXED = 1  /* FP32 operators and inner CG; FP64 state, FP64 outer
                    refinement residual, FP64 norms and divergence */
};

enum cfd_precond {
  CFD_PC_JACOBI = 0,   /* Jacobi-preconditioned CG (reference behaviour) */
  CFD_PC_LEARNED = 1,  /* Jacobi step + coarse-space correction + U-Net
                          correction in flexible CG, with Jacobi-PCG fallback
                          when it stalls */
  CFD_PC_TWOLEVEL = 2  /* Jacobi step + coarse-space correction (P Zc^-1 P^T,
                          Zc = P^T Z P on a coarse lattice of the structured
                          pressure grid) in CG: the learned preconditioner
                          without its network */
};

typedef struct cfd_ctx cfd_ctx;

typedef struct {
  int precision;     /* enum cfd_precision (default CFD_FP64) */
  int precond;       /* enum cfd_precond (default CFD_PC_JACOBI) */
  double cg_rtol;    /* stop when ||r||_2 <= cg_rtol*||b||_2 (default 1e-8) */
  int cg_maxit;      /* default 1000, as blascoCodinaHuerta.cpp:4013 */
  int cg_warm;       /* 0: x0 = 0 (MKL call site, blascoCodinaHuerta.cpp:4002);
                        1: x0 = previous solution (CUSP call site, CUDAcodes.cu:268) */
  int ngp_override;  /* 0: NGP from the deck; 8 or 27 overrides it */
  double inner_rtol; /* CFD_MIXED: inner FP32 solve tolerance (default 1e-4) */
  int max_outer;     /* CFD_MIXED: refinement sweeps (default 12) */
  int fcg_m;         /* CFD_PC_LEARNED: flexible-CG directions each new one is
                        orthogonalised against, 1..8 (default 4) */
  int fcg_net_iters; /* CFD_PC_LEARNED: the network's correction is applied in
                        the first fcg_net_iters iterations of each pressure
                        solve (of its first inner solve in CFD_MIXED), the
                        two-level part alone after them (0 = every iteration) */
  int deterministic; /* 1: element assembly and convection run one element
                        colour per launch (no two elements of a colour share
                        a node) with plain adds instead of FP64 atomics, so
                        repeated runs are bitwise identical, as the
                        reference's coloured assembly (CUDAcodes.cu:915-936);
                        0 (default): one launch over all elements, atomics */
} cfd_options;

typedef struct {
  int NE, NCN, NN, NNp, NGP, maxIter;
  long long nnzK, nnzG, nnzZ;
  int nBCnodes, monPoint, zeroPressureNode;
  double dt, t_ini, t_final, tolerance, convergence, density, viscosity;
  int timeN;
  double timeT;
} cfd_problem_info;

typedef struct {
  int iterations;   /* Krylov iterations (inner iterations in CFD_MIXED) */
  int outer;        /* refinement sweeps (CFD_MIXED), 0 otherwise */
  double relres;    /* final ||r||/||b|| (FP64 residual) */
  int status;       /* 0 converged, 1 iteration limit, 2 non-finite, 3 timeout */
  int fallback;     /* 1 when the learned preconditioner stalled and Jacobi took over */
} cfd_solve_stats;

typedef struct {
  int steps;             /* time steps run */
  long long subiters;    /* fractional-step sub-iterations run */
  long long cg_iters;    /* Krylov iterations over all solves */
  int steady;            /* 1 if the steady-state test fired */
  double maxAcc;         /* last max |Unp1-Un|/dt */
  int last_iter;         /* iteration index printed by the monitor (maxIter+1 if none converged) */
  int fallbacks;         /* pressure solves in which the learned preconditioner fell back to Jacobi */
} cfd_run_stats;

/* ---- context ---------------------------------------------------------- */

/* selectCUDAdevice, CUDAcodes.cu:126-154 (device < 0 picks the last device,
 * as the reference does). */
int cfd_create(cfd_ctx** out, int device);
void cfd_destroy(cfd_ctx* ctx);
const char* cfd_last_error(const cfd_ctx* ctx);
int cfd_abi_version(void);
void cfd_default_options(cfd_options* opt);
int cfd_set_options(cfd_ctx* ctx, const cfd_options* opt);

/* ---- problem set-up ---------------------------------------------------- */

/* readInputFile (blascoCodinaHuerta.cpp:528-725) followed by the mesh
 * preprocessing of blascoCodinaHuerta.cpp:732-2159 (hex27 node generation,
 * DOF maps, velocity-BC nodes, monitor node, CSR patterns), the basis set-up
 * of blascoCodinaHuerta.cpp:2166-2488, the initial condition of
 * applyBC_initial (blascoCodinaHuerta.cpp:4062-4110) and the device upload of
 * initializeAndAllocateGPU (CUDAcodes.cu:161-274). */
int cfd_load_inp(cfd_ctx* ctx, const char* path);

/* Same as cfd_load_inp from in-memory deck data (0-based ids):
 * coords NCN x 3, conn NE x 8, bcvals nBC x 3, velfaces nVelFaces x 3
 * (element, face 0..5, bc).  Header values come from info (NE, NCN, NGP,
 * maxIter, dt, t_ini, t_final, tolerance, convergence, density, viscosity,
 * zeroPressureNode) and monitor[3]. */
int cfd_load_mesh(cfd_ctx* ctx, const cfd_problem_info* info, const double* coords, const int* conn,
                  int nBC, const double* bcvals, int nVelFaces, const int* velfaces,
                  const double* monitor);

int cfd_info(const cfd_ctx* ctx, cfd_problem_info* info);

/* step0 (blascoCodinaHuerta.cpp:3127-3315) on the device: M row sums, K, G,
 * G^T assembled into their CSR slots, MdInv/MdOrigInv, and calculateZ_CUSP
 * (CUDAcodes.cu:281-411) including the Z[p][p] *= 1000 pin. */
int cfd_step0(cfd_ctx* ctx);

/* ---- one time step, stage by stage (timeLoop, blascoCodinaHuerta.cpp:2859-3094) */

/* timeN++, timeT += dt, UnpHalf_prev <- Un, Pnp1_prev <- Pn, Acc_prev <- 0
 * (blascoCodinaHuerta.cpp:2860-2881). */
int cfd_begin_step(cfd_ctx* ctx);
/* calculateMatrixAGPU, CUDAcodes.cu:906-939: R1 = -A(Un) UnpHalf_prev. */
int cfd_convect(cfd_ctx* ctx);
/* step1GPUpart, CUDAcodes.cu:946-973 (call cfd_convect first). */
int cfd_step1(cfd_ctx* ctx, int iter);
/* step2GPU, CUDAcodes.cu:980-1022 (pressure solve; stats may be NULL). */
int cfd_step2(cfd_ctx* ctx, int iter, cfd_solve_stats* st);
/* step3GPU, CUDAcodes.cu:1029-1060. */
int cfd_step3(cfd_ctx* ctx, int iter);
/* checkConvergenceGPU, CUDAcodes.cu:1084-1121; norms[0] = |dU|/|U|,
 * norms[1] = |dP|/|P| (may be NULL). */
int cfd_check_iter(cfd_ctx* ctx, double tol, int* converged, double* norms);
/* "Get ready for the next iteration" copies, blascoCodinaHuerta.cpp:2929-2932. */
int cfd_rotate(cfd_ctx* ctx);
/* calculate_KtimesAcc_prevGPU, CUDAcodes.cu:1067-1077. */
int cfd_k_times_acc(cfd_ctx* ctx);
/* checkConvergenceInTimeGPU, CUDAcodes.cu:1151-1178, with the CPU
 * semantics maxAcc = max |Unp1 - Un| / dt (blascoCodinaHuerta.cpp:3052-3060). */
int cfd_check_steady(cfd_ctx* ctx, double crit, double* maxAcc, int* steady);
/* Un <- Unp1, Pn <- Pnp1, blascoCodinaHuerta.cpp:3068-3081.  Called right
 * after cfd_rotate (a sub-iteration loop that ran out of iterations), it
 * still takes the last iterate, as the reference's copying rotation does. */
int cfd_end_step(cfd_ctx* ctx);

/* Whole time loop on the device with one small readback per sub-iteration:
 * nsteps > 0 runs that many steps, nsteps < 0 runs the reference's
 * while (timeT < t_final) loop.  Stops early on steady state. */
int cfd_run(cfd_ctx* ctx, int nsteps, cfd_run_stats* st);

/* ---- state and diagnostics --------------------------------------------- */

/* printMonitorDataGPU, CUDAcodes.cu:1128-1144, without the full-state copy:
 * out = {u, v, w, p} at node (node < 0: the deck's monitor node). */
int cfd_get_monitor(cfd_ctx* ctx, int node, double* out);
int cfd_download_state(cfd_ctx* ctx, double* U3NN, double* P);
int cfd_upload_state(cfd_ctx* ctx, const double* U3NN, const double* P);

enum cfd_vector_id {
  CFD_V_UN = 0, CFD_V_UNP1, CFD_V_UNP1_PREV, CFD_V_UNPHALF, CFD_V_UNPHALF_PREV, CFD_V_ACC,
  CFD_V_ACC_PREV, CFD_V_PN, CFD_V_PNP1, CFD_V_PNP1_PREV, CFD_V_PDOT, CFD_V_MDINV,
  CFD_V_MDORIGINV, CFD_V_KACC_PREV, CFD_V_R1, CFD_V_R2, CFD_V_R3, CFD_V_DIV
};
/* Any solver vector in the reference layout (3NN for velocity-sized, NNp
 * for pressure-sized; MdInv/MdOrigInv are returned as 3NN). CFD_V_DIV is the
 * discrete divergence G^T Unp1 (NNp), evaluated in FP64. */
int cfd_download_vector(cfd_ctx* ctx, int which, double* out);

enum cfd_matrix_id { CFD_M_K = 0, CFD_M_G = 1, CFD_M_GT = 2, CFD_M_Z = 3 };
/* nnz of a matrix (into *nnz) and, when the arrays are non-NULL, its CSR:
 * rowptr (nrows+1), col (nnz), val (nnz, or 3*nnz interleaved per entry
 * for G and G^T as [G1 G2 G3]).  FP64 values. */
int cfd_download_matrix(cfd_ctx* ctx, int which, long long* nnz, int* rowptr, int* col, double* val);

/* Solve Z x = rhs on the device with the configured method (the minimal
 * pressure-solve entry point); x holds the initial guess when cg_warm = 1. */
int cfd_pressure_solve(cfd_ctx* ctx, const double* rhs, double* x, cfd_solve_stats* st);

/* ---- files ---------------------------------------------------------------- */

/* createTecplot, blascoCodinaHuerta.cpp:4249-4482 (same text layout). */
int cfd_write_tecplot(cfd_ctx* ctx, const char* path, const char* title);
/* readRestartFile, blascoCodinaHuerta.cpp:4214-4242. */
int cfd_read_restart(cfd_ctx* ctx, const char* path);
/* Per-node Dirichlet values overriding the deck's constant BC values
 * (e.g. a parabolic duct inlet): n entries of node ids and 3n values. */
int cfd_set_bc_values(cfd_ctx* ctx, int n, const int* nodes, const double* uvw);

/* ---- learned preconditioner -------------------------------------------------
 * No counterpart in the reference.  A 3-level 3D convolutional U-Net on the
 * structured grid of pressure nodes maps a residual r (scaled to unit RMS)
 * to an approximation of the error Z^-1 r; with precond = CFD_PC_LEARNED the
 * pressure solve runs flexible CG with it (inner FP32 solves under
 * CFD_MIXED, FP64 otherwise) and falls back to Jacobi-PCG for the rest of
 * the solve when flexible CG stalls (cfd_solve_stats.fallback = 1).
 * Grids are nx x ny x nz voxels in x-fastest order with (n - 1) % 4 == 0 and
 * n >= 5 on every axis.  BF16 weights and activations, FP32 accumulation,
 * FP32 gradients and Adam state. */
typedef struct cfd_unet cfd_unet;
/* A network with seeded He-normal weights on the current CUDA device (device
 * < 0) or the given one. */
int cfd_unet_create(cfd_unet** out, int device, unsigned long long seed);
void cfd_unet_destroy(cfd_unet* net);
const char* cfd_unet_last_error(const cfd_unet* net);
long long cfd_unet_param_count(void);
/* FP32 parameters in layer order (weights [27][cin][cout], then bias). */
int cfd_unet_get_params(cfd_unet* net, float* out, long long n);
int cfd_unet_set_params(cfd_unet* net, const float* in, long long n);
/* Weight file: 8-byte tag "CFDUNET1", int64 count, count FP32 values. */
int cfd_unet_save(cfd_unet* net, const char* path);
int cfd_unet_read(cfd_unet* net, const char* path);
/* y = f(x) for one grid (x, y: nx*ny*nz floats; device pointers when
 * on_device != 0, host otherwise). */
int cfd_unet_forward(cfd_unet* net, const int dims[3], const float* x, float* y, int on_device);
/* Training loss of one sample, d = f(x) - t on the grid:
 *   w_l2 mean(d^2) + w_h1 (1/n) sum over axes of (d[i+e] - d[i])^2
 * over neighbour pairs (default w_l2 = 1, w_h1 = 0). */
int cfd_unet_set_loss(cfd_unet* net, float w_l2, float w_h1);
/* The loss of one sample and, when grad is non-NULL, its gradient with
 * respect to every parameter (host, cfd_unet_param_count()). */
int cfd_unet_gradient(cfd_unet* net, const int dims[3], const float* x, const float* t, int on_device,
                      float* loss, float* grad);
/* Forward convolutions on the tensor cores (tcgen05, the default where the
 * layer shape allows: stride 1, 16/32/64 input channels) or all on the
 * CUDA-core kernels (on = 0).  The backward pass always uses the CUDA-core
 * kernels. */
int cfd_unet_set_tensor_cores(cfd_unet* net, int on);
/* CFD_E_TIMEOUT if a bounded wait inside a tensor-core convolution gave up
 * since the network was created (the output of that launch is invalid). */
int cfd_unet_status(cfd_unet* net);
/* Stored tensor t (0..13) of the last forward pass as floats (n = voxels of
 * its level x channels, channels fastest); t = 13 is the FP32 output.  For
 * tests and inspection. */
int cfd_unet_tensor(cfd_unet* net, int t, float* out, long long n);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the mean loss of nb samples
 * stored one grid after another in x and t; *loss receives that mean. */
int cfd_unet_train_batch(cfd_unet* net, const int dims[3], int nb, const float* x, const float* t,
                         int on_device, float lr, float* loss);
/* Uses net as the context's learned preconditioner.  dims: the pressure-node
 * grid (product = NNp); p_of_vox (NNp entries, may be NULL = identity, i.e.
 * pressure node x + nx (y + ny z)) names the pressure node of each voxel.
 * The context keeps the pointer: net must stay alive, on the context's
 * device, until it is detached (net = NULL) or the context is destroyed. */
int cfd_unet_attach(cfd_ctx* ctx, cfd_unet* net, const int dims[3], const int* p_of_vox);
/* Reads a weight file into a network owned by the context and attaches it;
 * the grid is dims (NULL: a cube, NNp = m^3, identity numbering). */
int cfd_unet_load(cfd_ctx* ctx, const char* path, const int dims[3]);
/* r = rhs - Z x in FP64 (host buffers of NNp); *norm (may be NULL) = ||r||_2. */
int cfd_pressure_residual(cfd_ctx* ctx, const double* rhs, const double* x, double* r, double* norm);
/* Declares the structured grid of pressure nodes the coarse space and the
 * network work on: dims (product = NNp) and p_of_vox as in cfd_unet_attach.
 * Without it, a cube NNp = m^3 whose nodes are numbered x + m (y + m z) (node
 * coordinates checked) is used.  No counterpart in the reference (new
 * preconditioners). */
int cfd_set_pressure_grid(cfd_ctx* ctx, const int dims[3], const int* p_of_vox);
/* z = linear part of the configured preconditioner applied to r (FP64 host
 * buffers of NNp): D^-1 r for CFD_PC_JACOBI, D^-1 r + P Zc^-1 P^T r for
 * CFD_PC_TWOLEVEL and CFD_PC_LEARNED (the network's correction is not
 * included).  Builds the coarse space on first use.  No counterpart in the
 * reference (training targets of the network). */
int cfd_precond_apply(cfd_ctx* ctx, const double* r, double* z);

/* ---- timing, counters and self-tests ---------------------------------------- */

/* The context's CUDA stream (cudaStream_t) so callers can record events on it. */
void* cfd_stream(cfd_ctx* ctx);
/* Number of kernel launches the context issued since creation. */
long long cfd_launch_count(const cfd_ctx* ctx);

enum cfd_kernel_class {
  CFD_K_CONVECT = 0, CFD_K_STEP1, CFD_K_GT, CFD_K_PCG64, CFD_K_PCG32, CFD_K_RESID64, CFD_K_STEP3,
  CFD_K_SPMV_K3, CFD_K_PUPDATE, CFD_K_OTHER, CFD_K_UNET, CFD_K_FCG, CFD_K_COARSE, CFD_K_SPMV_Z, CFD_K_FCG2L,
  CFD_K_COUNT
};
/* Per-kernel-class CUDA-event timing on the context stream (on = 1 starts
 * and clears, 0 stops).  out receives CFD_K_COUNT triples
 * {launches, total milliseconds, Krylov iterations inside those launches}. */
int cfd_profile(cfd_ctx* ctx, int on);
int cfd_profile_read(cfd_ctx* ctx, double* out);
/* While profiling is on: the device time (milliseconds, summed over
 * launches) of the phases of the persistent two-level iteration (class
 * CFD_K_FCG2L).  out10[0..6], read in the first block of the launch:
 * restriction, coarse solve, preconditioned residual, neighbour wait,
 * structured SpMV with its dot products, reduction of the dots, update with
 * the (r,r) reduction (each phase's time includes the wait that ends it);
 * out10[7..9]: the smallest, mean and largest over the blocks of each
 * block's own SpMV time.  No counterpart in the reference. */
int cfd_profile_fcg2l(cfd_ctx* ctx, double* out10);

/* Inverse of a dense symmetric positive definite n x n matrix (host
 * buffers, row-major) computed on the given device in FP64: the blocked
 * Cholesky and inverse that build the coarse space of the two-level
 * preconditioners on the device.  CFD_E_NONFINITE when a pivot is not
 * positive.  No counterpart in the reference. */
int cfd_spd_inverse(int device, const double* a, int n, double* inv);

/* Galerkin coarse matrix Zc = P^T Z P of the two-level preconditioner built
 * on the given device, for a CSR matrix Z (host buffers, n rows, FP64) on a
 * structured grid dims (product = n, identity numbering x + nx (y + ny z)),
 * with a coarse lattice of about `spacing` fine steps (4 in the solver).
 * cd receives the coarse nodes per axis; zc (NULL: only the sizes) the
 * dense nc x nc matrix, nc = cd[0] cd[1] cd[2] (at most 6000), summed in
 * the order of cfdh_coarse_matrix and bit-identical to it.
 * CFD_E_BADINPUT when a row of Z reaches more than 3 coarse nodes per axis
 * (the solver then builds Zc on the host).  No counterpart in the
 * reference. */
int cfd_coarse_matrix(int device, const int dims[3], const int* rowptr, const int* col, const double* val,
                      double spacing, int* cd, double* zc);

/* Runs one small kernel whose bounded wait watches a flag nothing sets, with
 * the given limit in milliseconds.  Returns CFD_E_TIMEOUT when the wait gave
 * up as designed (the context stays usable), CFD_OK otherwise. */
int cfd_selftest_wait_timeout(cfd_ctx* ctx, int timeout_ms);

/* ---- pressure solve that allocates nothing ----------------------------------
 * No counterpart in the reference.  For callers that must not allocate or
 * free device memory while they solve (cudaFree synchronizes the whole
 * device; some hosts reserve all device memory up front in their own pool).
 * Jacobi-PCG (x0 = 0, stop at ||r||_2 <= rtol ||b||_2) on a CSR system whose
 * arrays -- rowptr (n+1), col and val (nnz), dinv = 1/diag (n), b (n) and the
 * output x (n) -- are DEVICE pointers owned by the caller, on the caller's
 * stream (NULL = legacy default stream) and the current device.  Work
 * vectors live in one static device array of fixed size (16.1 MiB, held by
 * every GPU that loads the library until exit), so n is limited to
 * CFD_NOALLOC_MAX_N; larger n returns CFD_E_BADARG with a message in errbuf.
 * The first call on a device looks the array up (once per device); make it
 * before any stream capture.  With CUDA's lazy module loading (the default)
 * that first call is also when the array is placed on the device, so it
 * needs 16.1 MiB free: a host that reserves device memory for its own pool
 * should make one warm-up call (any small system) before it does.  Calls share the array: calls that overlap on
 * the GPU race and must not be issued.  info (may be NULL) receives
 * {iterations, ||r||/||b||, status}; returns CFD_OK, CFD_E_NOCONV,
 * CFD_E_NONFINITE, CFD_E_TIMEOUT, CFD_E_BADARG or CFD_E_CUDA. */
#define CFD_NOALLOC_MAX_N 524288
int cfd_pcg_solve_noalloc(const int* rowptr, const int* col, const double* val, const double* dinv,
                          const double* b, double* x, int n, double rtol, int maxit, void* stream,
                          double* info, char* errbuf, int errlen);

/* ---- host-only preprocessing (no GPU needed) --------------------------------
 * The deck reader and mesh preprocessing of cfd_load_inp, exposed without a
 * device so callers can inspect the generated numbering and patterns. */
typedef struct cfd_host cfd_host;
/* readInputFile + setupNonCornerNodes + determineVelBCnodes +
 * findMonitorPoint + setupSparseM/G (blascoCodinaHuerta.cpp:528-2159). */
int cfdh_load(cfd_host** out, const char* path, char* errbuf, int errlen);
void cfdh_free(cfd_host* h);
/* sizes: NE NCN NN NNp nnzK nnzG nnzZ nBCnodes monPoint zeroPressureNode NGP maxIter */
int cfdh_sizes(const cfd_host* h, long long* out12);
int cfdh_get_ltog(const cfd_host* h, int* out);     /* NE x 27 */
int cfdh_get_coord(const cfd_host* h, double* out); /* NN x 3 */
int cfdh_get_bcnodes(const cfd_host* h, int* out);  /* nBCnodes x 2 (node, bc) */
/* Coarse space of the two-level preconditioner for a CSR matrix Z (n rows,
 * FP64 values) on a structured grid dims (product = n, identity numbering
 * x + nx (y + ny z)): cd receives the coarse nodes per axis; inv (NULL: only
 * the sizes) receives the nc x nc inverse of P^T Z P, nc = cd[0] cd[1] cd[2]
 * (at most 6000).  Host only; no counterpart in the reference. */
int cfdh_coarse_inverse(const int dims[3], const int* rowptr, const int* col, const double* val, int* cd,
                        double* inv);
/* The same coarse space's matrix Zc = P^T Z P itself (dense, symmetrised),
 * with the coarse spacing given (4 in the solver): the host counterpart of
 * cfd_coarse_matrix.  Host only; no counterpart in the reference. */
int cfdh_coarse_matrix(const int dims[3], const int* rowptr, const int* col, const double* val, double spacing,
                       int* cd, double* zc);
/* Element colouring of the deterministic mode (setupMeshColoring,
 * blascoCodinaHuerta.cpp:853-947): returns the number of colours C (or -1
 * beyond 64); order (NE, may be NULL) lists the elements colour by colour,
 * colour c owning order[off[c] .. off[c+1]) (off: C + 1 ints, may be NULL;
 * call once with NULLs to learn C). */
int cfdh_element_colors(const cfd_host* h, int* order, int* off);
/* which: 0 K (NN x NN), 1 G (NN x NNp), 2 G^T (NNp x NN), 3 Z (NNp x NNp) */
int cfdh_get_pattern(const cfd_host* h, int which, int* rowptr, int* col);
/* createTecplot layout (blascoCodinaHuerta.cpp:4249-4482) for given state. */
int cfdh_write_tecplot(const cfd_host* h, const double* U3NN, const double* P, const char* path,
                       const char* title);

#ifdef __cplusplus
}
#endif
#endif /* CFDFS_H */
