// TEST INFRASTRUCTURE ONLY (never part of the product): the reference's CUDA
// H.psi kernel source (cuda/hamiltonianMatrix.cuh:60-626), compiled as plain
// host C++ and run serially over every row, so that its index arithmetic can be
// checked on the CPU (under AddressSanitizer, against exact-size malloc'd maps
// built by the reference's own cuda/configurationsMap.cuh builders) and its
// output compared with the oracle, before the same kernel runs on a GPU.
//
// The kernel is a grid-stride loop over rows (i = blockIdx.x*blockDim.x +
// threadIdx.x; i += blockDim.x*gridDim.x), so a grid of one block of one thread
// visits every row exactly once.
//
//   refcuda_host N M in.bin out.bin
//   in.bin  : nc complex C, then M*M complex Ho (flat Ho[k + M*l]), then M^4 complex Hint
//   out.bin : nc complex H C
// Exit status 0 on success.
#include <cuda_runtime.h>
#include <cuComplex.h>

#include <stdio.h>
#include <stdlib.h>

// Host compilation of the kernel: the execution-space qualifiers become
// nothing and the launch coordinates become host variables.
#undef __global__
#define __global__
#undef __device__
#define __device__
static uint3 threadIdx, blockIdx;
static dim3 blockDim, gridDim;

#include "hamiltonianMatrix.cuh"

static int read_all(FILE *f, void *p, size_t bytes)
{
    return fread(p, 1, bytes, f) == bytes;
}

int main(int argc, char **argv)
{
    if (argc != 5) {
        fprintf(stderr, "usage: %s N M in.bin out.bin\n", argv[0]);
        return 2;
    }
    const int N = atoi(argv[1]), M = atoi(argv[2]);
    const int nc = NC(N, M);
    const size_t M2 = (size_t)M * M, M4 = M2 * M2;
    Carray C = (Carray)malloc(sizeof(cuDoubleComplex) * nc);
    Carray out = (Carray)malloc(sizeof(cuDoubleComplex) * nc);
    Carray Ho = (Carray)malloc(sizeof(cuDoubleComplex) * M2);
    Carray Hint = (Carray)malloc(sizeof(cuDoubleComplex) * M4);
    FILE *f = fopen(argv[3], "rb");
    if (!f || !read_all(f, C, sizeof(cuDoubleComplex) * nc) || !read_all(f, Ho, sizeof(cuDoubleComplex) * M2) ||
        !read_all(f, Hint, sizeof(cuDoubleComplex) * M4)) {
        fprintf(stderr, "cannot read %s\n", argv[3]);
        return 2;
    }
    fclose(f);

    Iarray NCmat = setupNCmat(N, M);
    Iarray IF = setupFocks(N, M);
    Iarray strideOT = iarrDef(nc), strideTT = iarrDef(nc);
    Iarray Map = OneOneMap(N, M, NCmat, IF);
    Iarray MapTT = TwoTwoMap(N, M, NCmat, IF, strideTT);
    Iarray MapOT = OneTwoMap(N, M, NCmat, IF, strideOT);

    blockIdx.x = threadIdx.x = 0;
    blockDim.x = gridDim.x = 1;
    applyHconf(N, M, Map, MapOT, MapTT, strideOT, strideTT, IF, C, Ho, Hint, out);

    f = fopen(argv[4], "wb");
    if (!f || fwrite(out, sizeof(cuDoubleComplex), nc, f) != (size_t)nc) {
        fprintf(stderr, "cannot write %s\n", argv[4]);
        return 2;
    }
    fclose(f);
    free(C); free(out); free(Ho); free(Hint);
    free(NCmat); free(IF); free(strideOT); free(strideTT); free(Map); free(MapTT); free(MapOT);
    return 0;
}
