/* Stand-in for MKL's mkl_blas.h (test infrastructure only).  The reference
 * includes it (blascoCodinaHuerta.cpp:102) but calls no dense BLAS routine. */
#ifndef REFSHIM_MKL_BLAS_H
#define REFSHIM_MKL_BLAS_H
#include "mkl_types.h"
#endif
