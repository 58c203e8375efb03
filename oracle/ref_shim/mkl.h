/* The MKL names the reference's cbm/cbm_extensions.cpp includes through
 * "mkl.h" -- TEST INFRASTRUCTURE ONLY (oracle/build_ref.py): the LP64 integer
 * type, the sparse BLAS declarations and cblas_saxpy.  Project-written from
 * MKL's published C API; declarations only. */
#ifndef CBM_REF_SHIM_MKL_H
#define CBM_REF_SHIM_MKL_H

#ifndef MKL_INT
#define MKL_INT int
#endif

#include "mkl_spblas.h"

#ifdef __cplusplus
extern "C" {
#endif
void cblas_saxpy(const MKL_INT n, const float a, const float* x, const MKL_INT incx, float* y, const MKL_INT incy);
int mkl_get_max_threads(void);
#ifdef __cplusplus
}
#endif
#endif
