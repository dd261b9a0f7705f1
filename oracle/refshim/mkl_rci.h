/* Stand-in for MKL's mkl_rci.h (test infrastructure only): the reverse-
 * communication conjugate-gradient interface the reference's pressure
 * solve drives (blascoCodinaHuerta.cpp:3981-4055).
 *
 * Protocol (Intel MKL reference, "RCI CG"): tmp holds 4n doubles.
 *   rci_request 1: the caller computes tmp[n..2n) = A * tmp[0..n)
 *   rci_request 2: the caller runs its own stopping test (ipar[9] != 0)
 *   rci_request 3: the caller applies the preconditioner,
 *                  tmp[3n..4n) = C^-1 * tmp[2n..3n)   (ipar[10] != 0)
 *   rci_request 0: converged;  -1: iteration limit reached;  < -1: error.
 * ipar[3] is the iteration count and ipar[4] its limit; ipar[7] enables the
 * limit test, ipar[8] the residual test dpar[4] <= dpar[3] with
 * dpar[2] = |r_0|^2, dpar[3] = dpar[0]*dpar[2] + dpar[1] and
 * dpar[4] = |r_k|^2 (squared 2-norms: dpar[0] = 1e-12 in the reference
 * means |r_k| <= 1e-6 |r_0|). */
#ifndef REFSHIM_MKL_RCI_H
#define REFSHIM_MKL_RCI_H
#include "mkl_types.h"
#ifdef __cplusplus
extern "C" {
#endif
void dcg_init(const MKL_INT* n, const double* x, const double* b, MKL_INT* rci_request,
              MKL_INT* ipar, double* dpar, double* tmp);
void dcg_check(const MKL_INT* n, const double* x, const double* b, MKL_INT* rci_request,
               MKL_INT* ipar, double* dpar, double* tmp);
void dcg(const MKL_INT* n, double* x, double* b, MKL_INT* rci_request, MKL_INT* ipar,
         double* dpar, double* tmp);
void dcg_get(const MKL_INT* n, const double* x, const double* b, const MKL_INT* rci_request,
             const MKL_INT* ipar, const double* dpar, const double* tmp, MKL_INT* itercount);
#ifdef __cplusplus
}
#endif
#endif
