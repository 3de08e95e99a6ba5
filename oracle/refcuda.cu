// TEST INFRASTRUCTURE ONLY (never part of the product): a harness around the
// reference's own CUDA H.psi kernel, so that tests can check it against the
// oracle and the B200 path and time it on the same GPU.
//
// The kernel and the host map builders come unmodified from the reference's
// cuda/ directory (included from REF/cuda by oracle/Makefile):
//   applyHconf               cuda/hamiltonianMatrix.cuh:60-626
//   setupNCmat, setupFocks   cuda/configurationsMap.cuh:245-356
//   OneOneMap                cuda/configurationsMap.cuh:358-414
//   TwoTwoMap, OneTwoMap     cuda/configurationsMap.cuh:416-650
// The launch shape is the reference driver's (cuda/performanceTest.cu:315-323):
// one thread per configuration, THREADS_PER_BLOCK = 256. The maps are int32 and
// flattened with int arithmetic, so only spaces whose largest map fits INT_MAX
// run (the reference aborts otherwise); refcuda_fits() reports that on the host.
//
// Layouts follow the kernel: Ho flat as Ho[k + M*l] (= the CPU reference's
// Ho[k][l]), Hint[k + s*M + q*M^2 + l*M^3], C and out as nc complex doubles.
#include "hamiltonianMatrix.cuh"

#include <stdint.h>
#include <string.h>

#define RC_API extern "C" __attribute__((visibility("default")))

namespace {

int64_t g_map_bytes = 0;

int fail(char *err, int len, const char *what, cudaError_t e)
{
    if (err && len > 0) snprintf(err, len, "%s: %s", what, cudaGetErrorString(e));
    return 1;
}

// Exact map sizes in int32 entries, from the occupation table, before any
// builder runs (the builders index with int and would overflow silently).
void map_sizes(int M, int64_t nc, const int *IF, int64_t *one, int64_t *ot, int64_t *tt)
{
    int64_t sot = 0, stt = 0;
    for (int64_t i = 0; i < nc; ++i) {
        int occ = 0, two = 0;
        for (int k = 0; k < M; ++k) {
            if (IF[k + i * M] > 0) occ++;
            if (IF[k + i * M] > 1) two++;
        }
        sot += (int64_t)two * M * M;
        stt += (int64_t)occ * (occ - 1) / 2 * M * M;
    }
    *one = nc * M * M;
    *ot = sot + (int64_t)M * M;       // allocation size used by cuda/performanceTest.cu:123
    *tt = stt;
}

}  // namespace

// 1 when every int32 index the reference kernel forms stays below INT_MAX.
RC_API int refcuda_fits(int N, int M)
{
    if (N < 1 || M < 1) return 0;
    long double n = 1;
    for (int i = 1; i <= N; ++i) n = n * (M - 1 + i) / i;
    if (n > INT_MAX) return 0;
    const int nc = NC(N, M);
    int *IF = setupFocks(N, M);
    int64_t one, ot, tt;
    map_sizes(M, nc, IF, &one, &ot, &tt);
    free(IF);
    return one < INT_MAX && ot < INT_MAX && tt < INT_MAX;
}

// Device bytes of the int32 tables the last refcuda_apply_h uploaded
// (IF, Map, MapOT, MapTT, strideOT, strideTT).
RC_API int64_t refcuda_map_bytes() { return g_map_bytes; }

// out = H C with the reference kernel. Runs it once untimed, then `reps` times
// back to back between CUDA events; *ms = average per launch. Returns 0 on
// success, 1 with a message in err otherwise.
RC_API int refcuda_apply_h(int N, int M, const double *C, const double *Ho, const double *Hint,
                           double *out, int reps, float *ms, char *err, int errlen)
{
    if (!refcuda_fits(N, M)) {
        if (err && errlen > 0) snprintf(err, errlen, "int32 maps overflow for N=%d M=%d", N, M);
        return 1;
    }
    const int nc = NC(N, M);
    int *NCmat = setupNCmat(N, M);
    int *IF = setupFocks(N, M);
    int *strideOT = iarrDef(nc), *strideTT = iarrDef(nc);
    int *Map = OneOneMap(N, M, NCmat, IF);
    int *MapTT = TwoTwoMap(N, M, NCmat, IF, strideTT);
    int *MapOT = OneTwoMap(N, M, NCmat, IF, strideOT);
    int64_t one, ot, tt;
    map_sizes(M, nc, IF, &one, &ot, &tt);

    int *d_IF = 0, *d_Map = 0, *d_OT = 0, *d_TT = 0, *d_sOT = 0, *d_sTT = 0;
    cuDoubleComplex *d_C = 0, *d_out = 0, *d_Ho = 0, *d_Hint = 0;
    cudaEvent_t e0 = 0, e1 = 0;
    int rc = 0;
    cudaError_t e;
    const size_t M2 = (size_t)M * M, M4 = M2 * M2;
#define RC_CHECK(x, what) do { e = (x); if (e != cudaSuccess) { rc = fail(err, errlen, what, e); goto done; } } while (0)
    RC_CHECK(cudaMalloc(&d_IF, sizeof(int) * (size_t)nc * M), "cudaMalloc IF");
    RC_CHECK(cudaMalloc(&d_Map, sizeof(int) * (size_t)one), "cudaMalloc Map");
    RC_CHECK(cudaMalloc(&d_OT, sizeof(int) * (size_t)ot), "cudaMalloc MapOT");
    RC_CHECK(cudaMalloc(&d_TT, sizeof(int) * (size_t)(tt > 0 ? tt : 1)), "cudaMalloc MapTT");
    RC_CHECK(cudaMalloc(&d_sOT, sizeof(int) * (size_t)nc), "cudaMalloc strideOT");
    RC_CHECK(cudaMalloc(&d_sTT, sizeof(int) * (size_t)nc), "cudaMalloc strideTT");
    RC_CHECK(cudaMalloc(&d_C, sizeof(cuDoubleComplex) * (size_t)nc), "cudaMalloc C");
    RC_CHECK(cudaMalloc(&d_out, sizeof(cuDoubleComplex) * (size_t)nc), "cudaMalloc out");
    RC_CHECK(cudaMalloc(&d_Ho, sizeof(cuDoubleComplex) * M2), "cudaMalloc Ho");
    RC_CHECK(cudaMalloc(&d_Hint, sizeof(cuDoubleComplex) * M4), "cudaMalloc Hint");
    RC_CHECK(cudaMemcpy(d_IF, IF, sizeof(int) * (size_t)nc * M, cudaMemcpyHostToDevice), "copy IF");
    RC_CHECK(cudaMemcpy(d_Map, Map, sizeof(int) * (size_t)one, cudaMemcpyHostToDevice), "copy Map");
    RC_CHECK(cudaMemcpy(d_OT, MapOT, sizeof(int) * (size_t)(ot - M2), cudaMemcpyHostToDevice), "copy MapOT");
    if (tt > 0) RC_CHECK(cudaMemcpy(d_TT, MapTT, sizeof(int) * (size_t)tt, cudaMemcpyHostToDevice), "copy MapTT");
    RC_CHECK(cudaMemcpy(d_sOT, strideOT, sizeof(int) * (size_t)nc, cudaMemcpyHostToDevice), "copy strideOT");
    RC_CHECK(cudaMemcpy(d_sTT, strideTT, sizeof(int) * (size_t)nc, cudaMemcpyHostToDevice), "copy strideTT");
    RC_CHECK(cudaMemcpy(d_C, C, sizeof(cuDoubleComplex) * (size_t)nc, cudaMemcpyHostToDevice), "copy C");
    RC_CHECK(cudaMemcpy(d_Ho, Ho, sizeof(cuDoubleComplex) * M2, cudaMemcpyHostToDevice), "copy Ho");
    RC_CHECK(cudaMemcpy(d_Hint, Hint, sizeof(cuDoubleComplex) * M4, cudaMemcpyHostToDevice), "copy Hint");
    g_map_bytes = (int64_t)sizeof(int) * ((int64_t)nc * M + one + ot + tt + 2 * (int64_t)nc);
    {
        const int blocks = (nc + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK;
        applyHconf<<<blocks, THREADS_PER_BLOCK>>>(N, M, d_Map, d_OT, d_TT, d_sOT, d_sTT, d_IF, d_C,
                                                  d_Ho, d_Hint, d_out);
        RC_CHECK(cudaGetLastError(), "launch applyHconf");
        RC_CHECK(cudaDeviceSynchronize(), "applyHconf");
        RC_CHECK(cudaEventCreate(&e0), "event");
        RC_CHECK(cudaEventCreate(&e1), "event");
        RC_CHECK(cudaEventRecord(e0), "event record");
        for (int r = 0; r < reps; ++r)
            applyHconf<<<blocks, THREADS_PER_BLOCK>>>(N, M, d_Map, d_OT, d_TT, d_sOT, d_sTT, d_IF, d_C,
                                                      d_Ho, d_Hint, d_out);
        RC_CHECK(cudaGetLastError(), "launch applyHconf");
        RC_CHECK(cudaEventRecord(e1), "event record");
        RC_CHECK(cudaEventSynchronize(e1), "applyHconf");
        float t = 0.f;
        RC_CHECK(cudaEventElapsedTime(&t, e0, e1), "elapsed");
        if (ms) *ms = reps > 0 ? t / reps : 0.f;
        RC_CHECK(cudaMemcpy(out, d_out, sizeof(cuDoubleComplex) * (size_t)nc, cudaMemcpyDeviceToHost), "copy out");
    }
#undef RC_CHECK
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_IF); cudaFree(d_Map); cudaFree(d_OT); cudaFree(d_TT); cudaFree(d_sOT); cudaFree(d_sTT);
    cudaFree(d_C); cudaFree(d_out); cudaFree(d_Ho); cudaFree(d_Hint);
    free(NCmat); free(IF); free(strideOT); free(strideTT); free(Map); free(MapTT); free(MapOT);
    return rc;
}
