/* mcpi_dropin -- the reference's own C interface, served by the B200 library.
 *
 * Same names, argument meaning, array layouts, ownership and error behaviour
 * as the functions defined in the reference's headers (andriati-alex/mcpi):
 * arrays returned by the set-up functions are malloc'd host memory the caller
 * free()s; outputs are caller-allocated; errors print a message and
 * exit(EXIT_FAILURE). Underneath, the tables are built and the operators are
 * applied on GPU `MCPI_DEVICE` (environment variable, default 0) through
 * libmcpi_b200.so; host vectors are copied to and from the device per call.
 * Maps passed back in (Map, MapOT, MapTT, strides) are accepted for
 * signature compatibility and not read: the device hashes every jump itself.
 *
 * include/dropin/ holds replacement configurationsMap.h, hamiltonianMatrix.h,
 * onebodyMatrix.h, twobodyMatrix.h and mkl.h that include this header, so the
 * reference drivers compile unmodified against it.
 */
#ifndef MCPI_DROPIN_H
#define MCPI_DROPIN_H

#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> mcpi_dropin_complex;
extern "C" {
#else
#include <complex.h>
typedef double complex mcpi_dropin_complex;
#endif

#if defined(__GNUC__)
#define MCPI_DROPIN_API __attribute__((visibility("default")))
#else
#define MCPI_DROPIN_API
#endif

typedef double *Rarray;
typedef mcpi_dropin_complex *Carray;
typedef mcpi_dropin_complex **Cmatrix;
typedef int *Iarray;

/* configurationsMap.h:46-116 */
MCPI_DROPIN_API Rarray rarrDef(unsigned int n);
MCPI_DROPIN_API Carray carrDef(unsigned int n);
MCPI_DROPIN_API Iarray iarrDef(unsigned int n);
MCPI_DROPIN_API Cmatrix cmatDef(unsigned int m, unsigned int n);
/* configurationsMap.h:120-141 */
MCPI_DROPIN_API long fac(int n);
/* configurationsMap.h:145-202 */
MCPI_DROPIN_API int NC(int N, int M);
/* configurationsMap.h:206-234 */
MCPI_DROPIN_API Iarray setupNCmat(int N, int M);
/* configurationsMap.h:238-269 */
MCPI_DROPIN_API void IndexToFock(int k, int N, int M, Iarray v);
/* configurationsMap.h:273-305 */
MCPI_DROPIN_API int FockToIndex(int N, int M, Iarray NCmat, Iarray v);
/* configurationsMap.h:309-344 */
MCPI_DROPIN_API Iarray setupFocks(int N, int M);
/* configurationsMap.h:348-417 */
MCPI_DROPIN_API Iarray OneOneMap(int N, int M, Iarray NCmat, Iarray IF);
/* configurationsMap.h:421-474 */
MCPI_DROPIN_API Iarray allocTwoTwoMap(int nc, int M, Iarray IF);
/* configurationsMap.h:478-613 */
MCPI_DROPIN_API Iarray TwoTwoMap(int N, int M, Iarray NCmat, Iarray IF, Iarray strideC);
/* configurationsMap.h:617-664 */
MCPI_DROPIN_API Iarray allocOneTwoMap(int nc, int M, Iarray IF);
/* configurationsMap.h:668-762 */
MCPI_DROPIN_API Iarray OneTwoMap(int N, int M, Iarray NCmat, Iarray IF, Iarray strideC);

/* hamiltonianMatrix.h:31-425 */
MCPI_DROPIN_API void applyHconf(int N, int M, Iarray NCmat, Iarray IF, Carray C, Cmatrix Ho,
                                Carray Hint, Carray out);
/* hamiltonianMatrix.h:431-887 */
MCPI_DROPIN_API void applyHconf_X(int N, int M, Iarray Map, Iarray MapOT, Iarray strideOT,
                                  Iarray NCmat, Iarray IF, Carray C, Cmatrix Ho, Carray Hint,
                                  Carray out);
/* hamiltonianMatrix.h:891-1425 */
MCPI_DROPIN_API void applyHconf_XX(int N, int M, Iarray Map, Iarray MapOT, Iarray MapTT,
                                   Iarray strideOT, Iarray strideTT, Iarray IF, Carray C,
                                   Cmatrix Ho, Carray Hint, Carray out);
/* hamiltonianMatrix.h:1431-1970 */
MCPI_DROPIN_API void applyHconf_omp(int N, int M, Iarray Map, Iarray MapOT, Iarray MapTT,
                                    Iarray strideOT, Iarray strideTT, Iarray IF, Carray C,
                                    Cmatrix Ho, Carray Hint, Carray out);

/* onebodyMatrix.h:34-110, 116-184, 190-251 */
MCPI_DROPIN_API void OBrho(int N, int M, Iarray NCmat, Carray C, Cmatrix rho);
MCPI_DROPIN_API void OBrho_X(int N, int M, Iarray NCmat, Iarray IF, Carray C, Cmatrix rho);
MCPI_DROPIN_API void OBrho_XM(int N, int M, Iarray Map, Iarray NCmat, Iarray IF, Carray C,
                              Cmatrix rho);

/* twobodyMatrix.h:38-496, 502-985, 991-1487 */
MCPI_DROPIN_API void TBrho(int N, int M, Iarray NCmat, Iarray IF, Carray C, Carray rho);
MCPI_DROPIN_API void TBrho_X(int N, int M, Iarray Map, Iarray MapOT, Iarray strideOT,
                             Iarray NCmat, Iarray IF, Carray C, Carray rho);
MCPI_DROPIN_API void TBrho_XX(int N, int M, Iarray Map, Iarray MapOT, Iarray MapTT,
                              Iarray strideOT, Iarray strideTT, Iarray NCmat, Iarray IF,
                              Carray C, Carray rho);

/* The LAPACKE routine groundStateLieb.c:435 calls (row-major, jobz 'V' or 'N'),
 * served by the library's implicit-QL tridiagonal solver. */
MCPI_DROPIN_API int LAPACKE_dstev(int matrix_layout, char jobz, int n, double *d, double *e,
                                  double *z, int ldz);

#ifdef __cplusplus
}
#endif

#endif /* MCPI_DROPIN_H */
