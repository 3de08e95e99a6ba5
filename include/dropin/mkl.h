/* Replacement for <mkl.h> as used by the reference's groundStateLieb.c: the
 * one LAPACKE routine it calls (LAPACKE_dstev, row-major) is served by
 * libmcpi_dropin.so's tridiagonal eigensolver. */
#ifndef MCPI_DROPIN_MKL_H
#define MCPI_DROPIN_MKL_H
#include "../mcpi_dropin.h"
#ifdef _OPENMP
#include <omp.h>
#endif
#ifndef LAPACK_ROW_MAJOR
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#endif
#endif
