// Implementations of the MKL and CSparse entry points that the reference's
// CPU solver (fractionalStep/Cpp/blascoCodinaHuerta.cpp, compiled without
// USECUDA) calls.  TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/fs_ref,
// the reference built from its own unmodified source so that its outputs can
// pin the oracle.  Nothing in the product links this file.
//
// Each routine follows the published contract of the library call it stands
// in for (Intel MKL reference manual: Sparse BLAS level 2 "mkl_?csrmv",
// "mkl_?csrsymv", "mkl_?csrsv" and the RCI CG solver "dcg"; T. A. Davis,
// Direct Methods for Sparse Linear Systems, SIAM 2006, chapter 2, for the
// CSparse routines).  The results are the same numbers up to the order of
// floating-point summation inside a row or column, which neither library
// documents.

#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cs.h"
#include "mkl_rci.h"
#include "mkl_service.h"
#include "mkl_spblas.h"

namespace {

// Threads of the routines below: the count mkl_set_num_threads asked for
// (the reference asks for 8, blascoCodinaHuerta.cpp:85, 404), capped by the
// OpenMP limits of the process (OMP_THREAD_LIMIT=1 gives one thread).
int g_threads = 0;

int nthreads() {
  const int t = g_threads > 0 ? g_threads : omp_get_max_threads();
  const int lim = omp_get_thread_limit();
  return t < lim ? t : lim;
}

inline bool is_char(const char* c, char lower) { return c && (*c == lower || *c == lower - 32); }

double dot(int n, const double* a, const double* b) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s) num_threads(nthreads())
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

// y[0..len) += sum of the per-thread partial vectors in thread order, where
// fill(buf, first, last) adds the contributions of rows [first, last) into
// its own zeroed buffer.  The row ranges are static blocks.
template <class F>
void scatter_rows(int rows, int len, double* y, F fill) {
  const int T = nthreads();
  if (T <= 1) {
    fill(y, 0, rows);
    return;
  }
  std::vector<double> part((size_t)T * len, 0.0);
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num(), nt = omp_get_num_threads();
    const int a = (int)((long)rows * t / nt), b = (int)((long)rows * (t + 1) / nt);
    fill(&part[(size_t)t * len], a, b);
#pragma omp barrier
#pragma omp for schedule(static)
    for (int c = 0; c < len; c++) {
      double acc = 0.0;
      for (int k = 0; k < nt; k++) acc += part[(size_t)k * len + c];
      y[c] += acc;
    }
  }
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- service
void mkl_set_dynamic(int) {}
void mkl_set_num_threads(int n) { g_threads = n; }
void MKL_Free_Buffers(void) {}

// ---------------------------------------------------------- Sparse BLAS
void mkl_dcsrmv(const char* transa, const MKL_INT* m, const MKL_INT* k, const double* alpha,
                const char* matdescra, const double* val, const MKL_INT* indx,
                const MKL_INT* pntrb, const MKL_INT* pntre, const double* x,
                const double* beta, double* y) {
  // Only general matrices occur at the reference's call sites.
  if (!is_char(&matdescra[0], 'g')) {
    std::fprintf(stderr, "refshim: mkl_dcsrmv supports matdescra[0] = 'g' only\n");
    std::abort();
  }
  const int base = is_char(&matdescra[3], 'f') ? 1 : 0;
  const int rows = *m, cols = *k;
  const double a = *alpha, b = *beta;
  if (is_char(transa, 'n')) {
#pragma omp parallel for schedule(static) num_threads(nthreads())
    for (int r = 0; r < rows; r++) {
      double s = 0.0;
      for (int q = pntrb[r] - base; q < pntre[r] - base; q++) s += val[q] * x[indx[q] - base];
      y[r] = (b == 0.0) ? a * s : a * s + b * y[r];
    }
  } else {
    // y (length k) := alpha * A^T x + beta * y
    for (int c = 0; c < cols; c++) y[c] = (b == 0.0) ? 0.0 : b * y[c];
    scatter_rows(rows, cols, y, [&](double* out, int first, int last) {
      for (int r = first; r < last; r++) {
        const double ax = a * x[r];
        for (int q = pntrb[r] - base; q < pntre[r] - base; q++) out[indx[q] - base] += val[q] * ax;
      }
    });
  }
}

void mkl_dcsrsymv(const char* uplo, const MKL_INT* m, const double* a, const MKL_INT* ia,
                  const MKL_INT* ja, const double* x, double* y) {
  // One-based three-array CSR holding one triangle of a symmetric matrix.
  const bool upper = is_char(uplo, 'u');
  const int n = *m;
  for (int r = 0; r < n; r++) y[r] = 0.0;
  // row r's stored entries give y[r] (a gather) and, off the diagonal, the
  // mirrored entries' contributions to y[c] (a scatter)
  scatter_rows(n, n, y, [&](double* out, int first, int last) {
    for (int r = first; r < last; r++) {
      double s = 0.0;
      for (int q = ia[r] - 1; q < ia[r + 1] - 1; q++) {
        const int c = ja[q] - 1;
        if (upper ? c < r : c > r) continue;  // outside the named triangle
        s += a[q] * x[c];
        if (c != r) out[c] += a[q] * x[r];
      }
      out[r] += s;
    }
  });
}

void mkl_dcsrsv(const char* transa, const MKL_INT* m, const double* alpha, const char* matdescra,
                const double* val, const MKL_INT* indx, const MKL_INT* pntrb,
                const MKL_INT* pntre, const double* x, double* y) {
  (void)transa;
  // The reference's descriptor is "dln" (diagonal, non-unit) and carries no
  // fourth (indexing) character; its arrays are one-based
  // (blascoCodinaHuerta.cpp:3497-3508), which the row pointers show.
  if (!is_char(&matdescra[0], 'd')) {
    std::fprintf(stderr, "refshim: mkl_dcsrsv supports diagonal matrices only\n");
    std::abort();
  }
  const int n = *m;
  const int base = (pntrb[0] == 1) ? 1 : 0;
#pragma omp parallel for schedule(static) num_threads(nthreads())
  for (int r = 0; r < n; r++) {
    double d = 0.0;
    for (int q = pntrb[r] - base; q < pntre[r] - base; q++)
      if (indx[q] - base == r) { d = val[q]; break; }
    y[r] = *alpha * x[r] / d;
  }
}

// ------------------------------------------------------------- RCI CG
// ipar[2] holds the stage of the reverse-communication loop:
//   1  first call: request A*x0 to form the initial residual
//   2  A*x0 is in tmp[n..): form r0, then request the preconditioner
//   3  z0 is in tmp[3n..): first direction p = z, request A*p
//   4  A*p is in tmp[n..): update x and r, run the stopping tests,
//      then request the preconditioner (or the user test first)
//   5  after the user test: request the preconditioner
//   6  z is in tmp[3n..): new direction, request A*p
// dpar[6] keeps (r, z) of the last direction between calls.
void dcg_init(const MKL_INT* n, const double* x, const double* b, MKL_INT* rci_request,
              MKL_INT* ipar, double* dpar, double* tmp) {
  (void)x; (void)b; (void)tmp;
  std::memset(ipar, 0, 128 * sizeof(MKL_INT));
  std::memset(dpar, 0, 128 * sizeof(double));
  ipar[0] = *n;
  ipar[1] = 6;
  ipar[2] = 1;
  ipar[3] = 0;
  ipar[4] = (*n < 150) ? *n : 150;
  ipar[5] = 1;
  ipar[6] = 1;
  ipar[7] = 1;
  ipar[8] = 0;
  ipar[9] = 1;
  ipar[10] = 0;
  dpar[0] = 1.0e-6;
  dpar[1] = 0.0;
  *rci_request = 0;
}

void dcg_check(const MKL_INT* n, const double* x, const double* b, MKL_INT* rci_request,
               MKL_INT* ipar, double* dpar, double* tmp) {
  (void)x; (void)b; (void)tmp;
  *rci_request = 0;
  if (*n <= 0 || ipar[0] != *n || ipar[4] <= 0 || dpar[0] < 0.0 || dpar[1] < 0.0) *rci_request = -1100;
}

void dcg(const MKL_INT* n_, double* x, double* b, MKL_INT* rci_request, MKL_INT* ipar,
         double* dpar, double* tmp) {
  const int n = *n_;
  double* p = tmp;
  double* Ap = tmp + n;
  double* r = tmp + 2 * (size_t)n;
  double* z = tmp + 3 * (size_t)n;
  const bool precond = ipar[10] != 0;
  for (;;) {
    switch (ipar[2]) {
      case 1:
        std::memcpy(p, x, sizeof(double) * n);
        ipar[2] = 2;
        *rci_request = 1;
        return;
      case 2:
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (int i = 0; i < n; i++) r[i] = b[i] - Ap[i];
        dpar[2] = dot(n, r, r);
        dpar[3] = dpar[0] * dpar[2] + dpar[1];
        dpar[4] = dpar[2];
        if (ipar[8] && dpar[4] <= dpar[3]) { *rci_request = 0; return; }
        ipar[2] = 3;
        if (precond) { *rci_request = 3; return; }
        std::memcpy(z, r, sizeof(double) * n);
        continue;
      case 3:
        std::memcpy(p, z, sizeof(double) * n);
        dpar[6] = dot(n, r, z);
        ipar[2] = 4;
        *rci_request = 1;
        return;
      case 4: {
        const double a = dpar[6] / dot(n, p, Ap);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (int i = 0; i < n; i++) {
          x[i] += a * p[i];
          r[i] -= a * Ap[i];
        }
        ipar[3] += 1;
        dpar[5] = dpar[4];
        dpar[4] = dot(n, r, r);
        if (ipar[8] && dpar[4] <= dpar[3]) { *rci_request = 0; return; }
        if (ipar[7] && ipar[3] >= ipar[4]) { *rci_request = -1; return; }
        if (ipar[9]) { ipar[2] = 5; *rci_request = 2; return; }
        ipar[2] = 5;
        continue;
      }
      case 5:
        ipar[2] = 6;
        if (precond) { *rci_request = 3; return; }
        std::memcpy(z, r, sizeof(double) * n);
        continue;
      case 6: {
        const double rz = dot(n, r, z);
        const double beta = rz / dpar[6];
        dpar[6] = rz;
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        ipar[2] = 4;
        *rci_request = 1;
        return;
      }
      default:
        *rci_request = -2;
        return;
    }
  }
}

void dcg_get(const MKL_INT* n, const double* x, const double* b, const MKL_INT* rci_request,
             const MKL_INT* ipar, const double* dpar, const double* tmp, MKL_INT* itercount) {
  (void)n; (void)x; (void)b; (void)rci_request; (void)dpar; (void)tmp;
  *itercount = ipar[3];
}

// ------------------------------------------------------------- CSparse
cs* cs_spalloc(int m, int n, int nzmax, int values, int triplet) {
  cs* A = (cs*)std::calloc(1, sizeof(cs));
  if (!A) return nullptr;
  A->m = m;
  A->n = n;
  A->nzmax = nzmax > 1 ? nzmax : 1;
  A->nz = triplet ? 0 : -1;
  A->p = (int*)std::malloc(sizeof(int) * (triplet ? A->nzmax : n + 1));
  A->i = (int*)std::malloc(sizeof(int) * A->nzmax);
  A->x = values ? (double*)std::malloc(sizeof(double) * A->nzmax) : nullptr;
  return A;
}

cs* cs_spfree(cs* A) {
  if (!A) return nullptr;
  std::free(A->p);
  std::free(A->i);
  std::free(A->x);
  std::free(A);
  return nullptr;
}

// Prefix sum of counts into column starts; leaves a copy of the starts in
// next[] to serve as insertion cursors.
static void starts_from_counts(int n, const std::vector<int>& count, int* start, std::vector<int>& next) {
  int run = 0;
  next.resize(n);
  for (int j = 0; j < n; j++) {
    start[j] = run;
    next[j] = run;
    run += count[j];
  }
  start[n] = run;
}

// Triplet -> compressed column; entries keep their triplet order inside a
// column (Davis, section 2.4).
cs* cs_compress(const cs* T) {
  if (!T || T->nz < 0) return nullptr;
  const int n = T->n, nz = T->nz;
  cs* C = cs_spalloc(T->m, n, nz, T->x != nullptr, 0);
  if (!C) return nullptr;
  std::vector<int> count(n, 0), next;
  for (int k = 0; k < nz; k++) count[T->p[k]]++;
  starts_from_counts(n, count, C->p, next);
  for (int k = 0; k < nz; k++) {
    const int q = next[T->p[k]]++;
    C->i[q] = T->i[k];
    if (C->x) C->x[q] = T->x[k];
  }
  return C;
}

// Compressed-column transpose; row indices of the result come out sorted
// because the source columns are visited in order (Davis, section 2.5).
cs* cs_transpose(const cs* A, int values) {
  if (!A || A->nz != -1) return nullptr;
  const int m = A->m, n = A->n;
  const int nnz = A->p[n];
  cs* C = cs_spalloc(n, m, nnz, values && A->x, 0);
  if (!C) return nullptr;
  std::vector<int> count(m, 0), next;
  for (int q = 0; q < nnz; q++) count[A->i[q]]++;
  starts_from_counts(m, count, C->p, next);
  for (int j = 0; j < n; j++)
    for (int q = A->p[j]; q < A->p[j + 1]; q++) {
      const int dst = next[A->i[q]]++;
      C->i[dst] = j;
      if (C->x) C->x[dst] = A->x[q];
    }
  return C;
}

// C = A*B column by column (Davis, section 2.8): column j of C accumulates
// B(k,j) * A(:,k) over the entries k of B(:,j) in their stored order into a
// dense work vector; a row enters C(:,j) in the order it is first reached.
// The result is trimmed so that nzmax equals the entry count.
cs* cs_multiply(const cs* A, const cs* B) {
  if (!A || !B || A->nz != -1 || B->nz != -1 || A->n != B->m) return nullptr;
  const int m = A->m, n = B->n;
  const bool vals = A->x && B->x;
  int cap = A->p[A->n] + B->p[n];
  cs* C = cs_spalloc(m, n, cap, vals, 0);
  if (!C) return nullptr;
  std::vector<int> mark(m, -1);
  std::vector<double> acc(vals ? m : 0);
  int nnz = 0;
  for (int j = 0; j < n; j++) {
    // worst case for this column: every row of A
    if (nnz + m > C->nzmax) {
      const int grow = 2 * C->nzmax + m;
      C->i = (int*)std::realloc(C->i, sizeof(int) * grow);
      if (vals) C->x = (double*)std::realloc(C->x, sizeof(double) * grow);
      C->nzmax = grow;
    }
    C->p[j] = nnz;
    const int col_begin = nnz;
    for (int q = B->p[j]; q < B->p[j + 1]; q++) {
      const int k = B->i[q];
      const double bkj = vals ? B->x[q] : 0.0;
      for (int t = A->p[k]; t < A->p[k + 1]; t++) {
        const int row = A->i[t];
        if (mark[row] != j) {
          mark[row] = j;
          C->i[nnz++] = row;
          if (vals) acc[row] = bkj * A->x[t];
        } else if (vals) {
          acc[row] += bkj * A->x[t];
        }
      }
    }
    if (vals)
      for (int q = col_begin; q < nnz; q++) C->x[q] = acc[C->i[q]];
  }
  C->p[n] = nnz;
  const int keep = nnz > 1 ? nnz : 1;
  C->i = (int*)std::realloc(C->i, sizeof(int) * keep);
  if (vals) C->x = (double*)std::realloc(C->x, sizeof(double) * keep);
  C->nzmax = nnz;
  return C;
}

int cs_print(const cs* A, int brief) {
  if (!A) { std::printf("(null)\n"); return 0; }
  if (A->nz < 0) {
    std::printf("%d-by-%d, nzmax: %d nnz: %d\n", A->m, A->n, A->nzmax, A->p[A->n]);
    for (int j = 0; j < A->n; j++) {
      std::printf("    col %d : locations %d to %d\n", j, A->p[j], A->p[j + 1] - 1);
      for (int q = A->p[j]; q < A->p[j + 1]; q++) {
        std::printf("      %d : %g\n", A->i[q], A->x ? A->x[q] : 1.0);
        if (brief && q > 20) { std::printf("  ...\n"); return 1; }
      }
    }
  } else {
    std::printf("triplet: %d-by-%d, nzmax: %d nnz: %d\n", A->m, A->n, A->nzmax, A->nz);
    for (int q = 0; q < A->nz; q++) {
      std::printf("    %d %d : %g\n", A->i[q], A->p[q], A->x ? A->x[q] : 1.0);
      if (brief && q > 20) { std::printf("  ...\n"); return 1; }
    }
  }
  return 1;
}

}  // extern "C"
