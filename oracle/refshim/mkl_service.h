/* Stand-in for MKL's mkl_service.h (test infrastructure only): the service
 * calls the reference makes (blascoCodinaHuerta.cpp:403-404, 4009-4043). */
#ifndef REFSHIM_MKL_SERVICE_H
#define REFSHIM_MKL_SERVICE_H
#include "mkl_types.h"
#ifdef __cplusplus
extern "C" {
#endif
void mkl_set_dynamic(int flag);
void mkl_set_num_threads(int n);
void MKL_Free_Buffers(void);
#ifdef __cplusplus
}
#endif
#endif
