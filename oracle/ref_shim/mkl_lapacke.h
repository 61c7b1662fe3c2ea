/* Stand-in for <mkl_lapacke.h> when building the reference's GPU code as a
 * test oracle: MKL is not installed, so LAPACKE_dstedc is forwarded to the
 * LAPACKE of the OpenBLAS that ships with scipy (32-bit lapack_int). */
#pragma once
#include <stdint.h>
typedef int32_t lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#ifdef __cplusplus
extern "C" {
#endif
lapack_int scipy_LAPACKE_dstedc(int matrix_layout, char compz, lapack_int n, double* d, double* e,
                                double* z, lapack_int ldz);
#ifdef __cplusplus
}
#endif
#define LAPACKE_dstedc scipy_LAPACKE_dstedc
