// H.psi without any allocation: mcpi_apply_h_static.
//
// Some callers cannot allocate device memory at the point where they need
// H.psi: a host that has handed (nearly) all of the GPU's memory to its own
// pool allocator -- PyTorch's caching allocator does this -- can see a foreign
// cudaMalloc fail even though its pool has room, and a latency-bound loop
// cannot absorb the device-wide synchronisation that cudaMalloc/cudaFree may
// imply. For them this entry point runs the same two H.psi kernels as
// mcpi_apply_h, but every piece of scratch they need (binomial and square-root
// tables, the pair operator, and the P x NC(N-2,M) intermediate E) is carved
// out of one fixed array compiled into the library, g_scratch below. The
// caller supplies the input and output vectors; nothing is allocated on the
// device or on the host heap on the success path.
//
// Limits and sharing: g_scratch holds kScratchBytes (32 MiB) on every GPU that
// loads the library, for the life of the process. Requests whose tables and E
// do not fit are rejected with MCPI_ERR_RANGE before anything is enqueued
// (at M = 10 that admits N <= 10; see mcpi_apply_h_static in mcpi_b200.h).
// All calls on a device share the one array and it keeps the last call's
// contents; every region a call's kernels read is rewritten by that call
// first (E completely, by the first kernel), so nothing needs clearing, but
// two calls whose work overlaps on the GPU (different streams, or different
// host threads without ordering) race on it and must be serialised by the
// caller.
//
// Set-up: the first call on each device looks up the device address of
// g_scratch with cudaGetSymbolAddress (host code cannot use the symbol itself
// as a device pointer) while that device is current, and caches it; make that
// first call before any stream capture begins.
//
// Not for stream capture: each call copies its freshly folded tables from
// buffers on the calling thread's stack with pageable cudaMemcpyAsync, which a
// captured graph could not replay (the buffers are gone by then). A call on a
// stream that is capturing -- or on the legacy default stream while another
// stream captures -- returns MCPI_ERR_ARG before it enqueues anything, so the
// caller's capture stays intact.
//
// Host stack: the folded pair matrix (P*P complex, compacted in place into
// the nonzero values), its column indices and the binomial tables take about
// 58 KB of the calling thread's stack at M = 10; threads with small stacks
// (some worker pools, musl's 128 KB default) must leave room for that.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>

#include "../../include/mcpi_b200.h"
#include "fock.cuh"
#include "kernels.h"
#include "pairfold.h"

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxStaticM = 10;
constexpr int kMaxStaticP = kMaxStaticM * (kMaxStaticM + 1) / 2;
constexpr int kMaxStaticWs = 64 + 3;   // N <= 64
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_ptr[kMaxDevices];   // device address of g_scratch per device ordinal

using cplx = std::complex<double>;

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

int64_t binom64(int n, int k)   // exact for the small arguments admitted here
{
    if (k < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 r = 1;
    for (int i = 1; i <= k; ++i) r = r * (unsigned)(n - k + i) / (unsigned)i;
    return (int64_t)r;
}

}  // namespace

extern "C" MCPI_API int mcpi_apply_h_static(int N, int M, const double *h_Ho, const double *h_Hint,
                                             int variant, const void *d_C, void *d_out, void *stream)
{
    if (!h_Ho || !h_Hint || !d_C || !d_out || d_C == d_out) return MCPI_ERR_ARG;
    if (variant != MCPI_VARIANT_MAPS && variant != MCPI_VARIANT_HASH) return MCPI_ERR_ARG;
    if (N < 0 || M < 1) return MCPI_ERR_ARG;
    if (M > kMaxStaticM || N + 3 > kMaxStaticWs) return MCPI_ERR_RANGE;
    const int P = M * (M + 1) / 2, ws = N + 3;
    const int64_t nc = binom64(N + M - 1, N);
    const int64_t nc2 = N >= 2 ? binom64(N - 2 + M - 1, N - 2) : 0;
    const int64_t nc1 = N >= 1 ? binom64(N - 1 + M - 1, N - 1) : 0;
    // scratch layout (256-byte aligned regions)
    const size_t oW = 0, oSq = oW + up256(sizeof(uint32_t) * (M > 1 ? M - 1 : 1) * ws);
    const size_t oRow = oSq + up256(sizeof(double) * ws);
    const size_t oCol = oRow + up256(sizeof(int) * (P + 1));
    const size_t oVal = oCol + up256(sizeof(uint16_t) * P * P);
    const size_t oHd = oVal + up256(sizeof(double2) * P * P);
    const size_t oHf = oHd + up256(sizeof(double2) * M);
    const size_t oE = oHf + up256(sizeof(double2) * M * M);
    const size_t need = oE + sizeof(double2) * (size_t)P * (size_t)nc2;
    if (need > kScratchBytes || nc >= ((int64_t)1 << 31)) return MCPI_ERR_RANGE;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        // refuse capture before touching anything else (see the file comment);
        // an error from the query itself (the legacy stream while another
        // stream captures globally) counts as capturing
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return MCPI_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MCPI_ERR_CUDA;
    unsigned char *base;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return MCPI_ERR_CUDA;
            g_scratch_ptr[dev] = p;
        }
        base = static_cast<unsigned char *>(g_scratch_ptr[dev]);
    }

    // host-side tables, on the stack (about 58 KB at M = 10)
    uint32_t W[(kMaxStaticM - 1) * kMaxStaticWs];
    double sq[kMaxStaticWs];
    int rowptr[kMaxStaticP + 1];
    uint16_t col[kMaxStaticP * kMaxStaticP];
    cplx Ht[kMaxStaticP * kMaxStaticP], hd[kMaxStaticM];
    for (int i = 0; i + 1 < M; ++i)
        for (int p = 0; p < ws; ++p) W[i * ws + p] = (uint32_t)binom64(p + i, i + 1);
    for (int n = 0; n < ws; ++n) sq[n] = std::sqrt((double)n);
    const cplx *Ho = reinterpret_cast<const cplx *>(h_Ho);
    const cplx *Hint = reinterpret_cast<const cplx *>(h_Hint);
    mcpi::fold_pair_matrix(N, M, Ho, Hint, variant == MCPI_VARIANT_HASH, Ht);
    // compressed rows, compacted in place: entry nnz is written only after
    // entry a * P + b >= nnz has been read
    cplx *val = Ht;
    int nnz = 0;
    for (int a = 0; a < P; ++a) {
        rowptr[a] = nnz;
        for (int b = 0; b < P; ++b) {
            const cplx h = Ht[a * P + b];
            if (h != cplx(0.0, 0.0)) {
                col[nnz] = (uint16_t)b;
                val[nnz++] = h;
            }
        }
    }
    rowptr[P] = nnz;
    for (int k = 0; k < M; ++k) hd[k] = Ho[k * M + k];

    cudaError_t e = cudaSuccess;
    auto put = [&](size_t off, const void *src, size_t bytes) {
        if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st);
    };
    // pageable sources: each copy has consumed its stack buffer when it returns
    put(oW, W, sizeof(uint32_t) * (M > 1 ? M - 1 : 0) * ws);
    put(oSq, sq, sizeof(double) * ws);
    put(oRow, rowptr, sizeof(int) * (P + 1));
    put(oCol, col, sizeof(uint16_t) * nnz);
    put(oVal, val, sizeof(double2) * nnz);
    put(oHd, hd, sizeof(double2) * M);
    put(oHf, h_Ho, sizeof(double2) * M * M);
    if (e != cudaSuccess) return MCPI_ERR_CUDA;

    mcpi::Space sp{};
    sp.N = N;
    sp.M = M;
    sp.wstride = ws;
    sp.nc = (uint32_t)nc;
    sp.nc1 = (uint32_t)nc1;
    sp.nc2 = (uint32_t)nc2;
    const mcpi::SpaceTables tb{reinterpret_cast<const uint32_t *>(base + oW),
                               reinterpret_cast<const double *>(base + oSq)};
    mcpi::PairOp op{};
    op.rowptr = reinterpret_cast<const int *>(base + oRow);
    op.col = reinterpret_cast<const uint16_t *>(base + oCol);
    op.val = reinterpret_cast<const double2 *>(base + oVal);
    op.hdiag = reinterpret_cast<const double2 *>(base + oHd);
    op.hfull = reinterpret_cast<const double2 *>(base + oHf);
    op.nnz = nnz;
    op.hblk = nullptr;
    op.nhblk = 0;
    op.create_form = 0;
    op.status = nullptr;
    const mcpi::BlockOp bo{nullptr, 0};
    e = mcpi::launch_apply_h(sp, tb, op, bo, static_cast<const double2 *>(d_C),
                             reinterpret_cast<double2 *>(base + oE), static_cast<double2 *>(d_out), st);
    return e == cudaSuccess ? MCPI_OK : MCPI_ERR_CUDA;
}
