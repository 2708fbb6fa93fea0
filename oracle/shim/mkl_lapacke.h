/* Test-infrastructure shim: routes the three LAPACKE calls the reference
 * makes (multiconfig_lanczos.c:143, coefficients_integration.c:111,
 * lapack_interface.c:41,83,121) to the LP64 LAPACKE bundled with scipy
 * (libscipy_openblas, symbols prefixed `scipy_`). */
#ifndef ORACLE_SHIM_MKL_LAPACKE_H
#define ORACLE_SHIM_MKL_LAPACKE_H
#include "mkl_types.h"

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

int scipy_LAPACKE_dstev(int layout, char jobz, int n, double* d, double* e,
                        double* z, int ldz);
int scipy_LAPACKE_zheev(int layout, char jobz, char uplo, int n,
                        MKL_Complex16* a, int lda, double* w);
int scipy_LAPACKE_zhesv(int layout, char uplo, int n, int nrhs,
                        MKL_Complex16* a, int lda, int* ipiv, MKL_Complex16* b,
                        int ldb);

#define LAPACKE_dstev scipy_LAPACKE_dstev
#define LAPACKE_zheev scipy_LAPACKE_zheev
#define LAPACKE_zhesv scipy_LAPACKE_zhesv
#endif
