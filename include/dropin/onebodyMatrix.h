/* Replacement for the reference's onebodyMatrix.h: declares the same functions, which
 * libmcpi_dropin.so implements on the GPU (see ../mcpi_dropin.h). A driver that
 * includes "onebodyMatrix.h" compiles unmodified with -I <this directory> and links
 * -lmcpi_dropin -lmcpi_b200. */
#ifndef MCPI_DROPIN_onebodyMatrix_H
#define MCPI_DROPIN_onebodyMatrix_H
#include "../mcpi_dropin.h"
#ifdef _OPENMP
#include <omp.h>
#endif
#endif
