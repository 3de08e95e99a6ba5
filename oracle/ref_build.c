/* Translation unit that compiles the reference's own C sources, unmodified and
 * in place, into the test oracle library oracle/_ref/libmcpi_ref.so (see
 * oracle/Makefile). Nothing here is product code and nothing is copied: the
 * includes below read the reference files where they lie (-I <reference>).
 *
 *   configurationsMap.h  NC, setupNCmat, IndexToFock, FockToIndex, setupFocks,
 *                        OneOneMap, OneTwoMap, TwoTwoMap (+ alloc*)
 *   hamiltonianMatrix.h  applyHconf, applyHconf_X, applyHconf_XX, applyHconf_omp
 *   onebodyMatrix.h      OBrho, OBrho_X, OBrho_XM
 *   twobodyMatrix.h      TBrho, TBrho_X, TBrho_XX
 *   groundStateLieb.c    carrDot, carrMod, setupHo, setupHint, lanczos, ground
 *                        (its main() is renamed so the file links as a library;
 *                        <mkl.h> resolves to oracle/shim/mkl.h)
 */
#include "onebodyMatrix.h"
#include "twobodyMatrix.h"
#include "hamiltonianMatrix.h"

#define main mcpi_ref_groundStateLieb_main
#include "groundStateLieb.c"
#undef main
