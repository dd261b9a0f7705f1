/* Stand-in for Intel MKL's mkl_types.h, written for this repository so that
 * the reference's CPU solver (fractionalStep/Cpp/blascoCodinaHuerta.cpp)
 * compiles without MKL.  TEST INFRASTRUCTURE ONLY: it builds the checker
 * oracle/_ref/fs_ref and nothing in the product links it.
 * LP64 interface: MKL_INT is a 32-bit int, as with -lmkl_intel_lp64
 * (fractionalStep/Cpp/linuxCompile.txt:9-13). */
#ifndef REFSHIM_MKL_TYPES_H
#define REFSHIM_MKL_TYPES_H
#define MKL_INT int
#endif
