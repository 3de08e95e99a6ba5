/* Stand-in for <mkl.h> used ONLY to compile the reference's groundStateLieb.c
 * into the test oracle (oracle/_ref). It declares the single LAPACKE routine
 * that file calls (groundStateLieb.c:435, LAPACKE_dstev with ROW_MAJOR and
 * jobz='V'); the definition is the oracle's own cyclic-Jacobi eigensolver in
 * oracle/lapacke_jacobi.c. Test infrastructure, never linked into the product. */
#ifndef MCPI_ORACLE_MKL_SHIM_H
#define MCPI_ORACLE_MKL_SHIM_H

#ifdef _OPENMP
#include <omp.h>
#endif

typedef int lapack_int;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int LAPACKE_dstev(int matrix_layout, char jobz, lapack_int n,
                         double *d, double *e, double *z, lapack_int ldz);

#endif
