/* Stand-in for MKL's mkl_spblas.h (test infrastructure only): the three
 * classic Sparse BLAS routines of the reference's CPU path.
 *   mkl_dcsrmv   y := alpha*op(A)*x + beta*y, A an m-by-k CSR matrix given
 *                as (val, indx, pntrb, pntre); matdescra[0] 'g' (general),
 *                matdescra[3] 'c' zero-based / 'f' one-based; op = A for
 *                transa 'n', A^T for 't'.  With beta = 0, y is not read.
 *                (blascoCodinaHuerta.cpp:3006-3022, 3746-3758, 3865-3868, 3933-3935)
 *   mkl_dcsrsymv y := A*x, A symmetric m-by-m with only the triangle named
 *                by uplo stored, three-array CSR, one-based.
 *                (blascoCodinaHuerta.cpp:4036)
 *   mkl_dcsrsv   y := alpha*inv(T)*x; the reference passes matdescra "dln"
 *                (diagonal matrix, non-unit), i.e. division by the stored
 *                diagonal.  (blascoCodinaHuerta.cpp:4039) */
#ifndef REFSHIM_MKL_SPBLAS_H
#define REFSHIM_MKL_SPBLAS_H
#include "mkl_types.h"
#ifdef __cplusplus
extern "C" {
#endif
void mkl_dcsrmv(const char* transa, const MKL_INT* m, const MKL_INT* k, const double* alpha,
                const char* matdescra, const double* val, const MKL_INT* indx,
                const MKL_INT* pntrb, const MKL_INT* pntre, const double* x,
                const double* beta, double* y);
void mkl_dcsrsymv(const char* uplo, const MKL_INT* m, const double* a, const MKL_INT* ia,
                  const MKL_INT* ja, const double* x, double* y);
void mkl_dcsrsv(const char* transa, const MKL_INT* m, const double* alpha, const char* matdescra,
                const double* val, const MKL_INT* indx, const MKL_INT* pntrb,
                const MKL_INT* pntre, const double* x, double* y);
#ifdef __cplusplus
}
#endif
#endif
