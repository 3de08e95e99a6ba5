// C ABI of libmcpi_b200.so: space contexts, the pair-operator planner and the
// host side of the Lanczos solver. Declarations: include/mcpi_b200.h.
#include "../../include/mcpi_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fock.cuh"
#include "kernels.h"
#include "pairfold.h"
#include "space.h"

namespace mcpi {
int tridiag_eig(int n, double *d, const double *e, double *z);
}

using mcpi::DevPairOp;
using mcpi::PairOp;
using mcpi::Space;
using mcpi::SpaceTables;
using cplx = std::complex<double>;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t _e = (call);                                                           \
        if (_e != cudaSuccess)                                                             \
            return fail(_e == cudaErrorMemoryAllocation ? MCPI_ERR_NOMEM : MCPI_ERR_CUDA,  \
                        "%s failed: %s", #call, cudaGetErrorString(_e));                   \
    } while (0)

#define CHECK_ARG(cond, msg)                                   \
    do {                                                       \
        if (!(cond)) return fail(MCPI_ERR_ARG, "%s", (msg));   \
    } while (0)

// Exact binomial C(n, k) in 128 bits (n small enough for every use here).
unsigned __int128 binom128(int64_t n, int64_t k)
{
    if (k < 0 || n < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 r = 1;
    for (int64_t i = 1; i <= k; ++i) r = r * (unsigned __int128)(n - k + i) / (unsigned __int128)i;
    return r;
}

int64_t nc_exact(int N, int M)  // -1 when it does not fit in 63 bits
{
    if (N < 0 || M < 1) return 0;
    unsigned __int128 r = binom128((int64_t)N + M - 1, N);
    return r > (unsigned __int128)INT64_MAX ? -1 : (int64_t)r;
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};


}  // namespace


namespace {

void free_op(DevPairOp &o)
{
    cudaFree(o.hblk);
    cudaFree(o.prog);
    cudaFree(o.rowptr);
    cudaFree(o.col);
    cudaFree(o.val);
    cudaFree(o.hdiag);
    cudaFree(o.hfull);
    cudaFree(o.hdense);
    o = DevPairOp{};
}

// Pair matrix Ht of the two-body sum plus the folded off-diagonal one-body
// part (pairfold.h: rule by rule as hamiltonianMatrix.h:976-1418 reads Hint).
std::vector<cplx> build_pair_matrix(int N, int M, const cplx *Ho, const cplx *Hint, int variant)
{
    const int P = M * (M + 1) / 2;
    std::vector<cplx> Ht((size_t)P * P);
    mcpi::fold_pair_matrix(N, M, Ho, Hint, variant == MCPI_VARIANT_HASH, Ht.data());
    return Ht;
}

// Decomposes Ht into independent blocks (connected components of the
// bipartite row/column graph of its nonzeros) and packs them for the
// block-sparse kernel (layout in kernels.h, BlockOp). Empty vector when some
// block has more than kBlockCols columns or the packed form is too large.
std::vector<int> pack_blocks(const std::vector<cplx> &Ht, int P, int M)
{
    std::vector<int> parent(2 * P);
    for (int x = 0; x < 2 * P; ++x) parent[x] = x;
    auto find = [&](int x) {
        while (parent[x] != x) x = parent[x] = parent[parent[x]];
        return x;
    };
    for (int a = 0; a < P; ++a)
        for (int b = 0; b < P; ++b)
            if (Ht[(size_t)a * P + b] != cplx(0.0, 0.0)) parent[find(a)] = find(P + b);
    std::vector<std::vector<int>> brow(2 * P), bcol(2 * P);
    for (int a = 0; a < P; ++a) brow[find(a)].push_back(a);
    for (int b = 0; b < P; ++b) bcol[find(P + b)].push_back(b);
    std::vector<int> roots;
    for (int x = 0; x < 2 * P; ++x)
        if (!brow[x].empty()) {
            if ((int)bcol[x].size() > mcpi::kBlockCols) return {};
            roots.push_back(x);
        }
    std::vector<int> qs(P), ls(P);
    for (int q = 0; q < M; ++q)
        for (int l = q; l < M; ++l) {
            qs[mcpi::pair_index(q, l, M)] = q;
            ls[mcpi::pair_index(q, l, M)] = l;
        }
    const int nb = (int)roots.size();
    std::vector<int> hdr, cols, rows;
    std::vector<cplx> vals;
    for (int x : roots) {
        hdr.push_back((int)cols.size());
        hdr.push_back((int)bcol[x].size());
        hdr.push_back((int)rows.size());
        hdr.push_back((int)brow[x].size());
        hdr.push_back((int)vals.size());
        for (int b : bcol[x]) cols.push_back(qs[b] | (ls[b] << 8));
        for (int a : brow[x]) {
            rows.push_back(a);
            for (int b : bcol[x]) vals.push_back(Ht[(size_t)a * P + b]);
        }
    }
    std::vector<int> prog = {nb, (int)cols.size(), (int)rows.size(), (int)vals.size()};
    prog.insert(prog.end(), hdr.begin(), hdr.end());
    prog.insert(prog.end(), cols.begin(), cols.end());
    prog.insert(prog.end(), rows.begin(), rows.end());
    while ((prog.size() * 4) % 16) prog.push_back(0);
    const size_t off = prog.size();
    prog.resize(off + vals.size() * 4);
    std::memcpy(prog.data() + off, vals.data(), vals.size() * sizeof(cplx));
    if (prog.size() * 4 > 96 * 1024) return {};
    return prog;
}

// Momentum-block packing (layout in kernels.h, PairOp::hblk): empty when Ht
// couples two pairs of different total q + l.
std::vector<cplx> pack_momentum(const std::vector<cplx> &Ht, int P, int M)
{
    for (int k = 0; k < M; ++k)
        for (int s = k; s < M; ++s)
            for (int q = 0; q < M; ++q)
                for (int l = q; l < M; ++l)
                    if (k + s != q + l &&
                        Ht[(size_t)mcpi::pair_index(k, s, M) * P + mcpi::pair_index(q, l, M)] != cplx(0.0, 0.0))
                        return {};
    std::vector<cplx> out;
    for (int K = 0; K <= 2 * M - 2; ++K) {
        const int qlo = K - (M - 1) > 0 ? K - (M - 1) : 0, qhi = K / 2;
        for (int r = qlo; r <= qhi; ++r)
            for (int c = qlo; c <= qhi; ++c)
                out.push_back(Ht[(size_t)mcpi::pair_index(r, K - r, M) * P + mcpi::pair_index(c, K - c, M)]);
    }
    return out;
}

int upload_op(mcpi_space_s *sp, DevPairOp &op, const std::vector<cplx> &Ht, const cplx *hdiag,
              const cplx *hfull)
{
    const int P = sp->P, M = sp->M;
    std::vector<int> rowptr(P + 1, 0);
    std::vector<uint16_t> col;
    std::vector<cplx> val;
    for (int a = 0; a < P; ++a) {
        for (int b = 0; b < P; ++b) {
            const cplx h = Ht[(size_t)a * P + b];
            if (h != cplx(0.0, 0.0)) {
                col.push_back((uint16_t)b);
                val.push_back(h);
            }
        }
        rowptr[a + 1] = (int)col.size();
    }
    free_op(op);
    const size_t nnz = col.size() ? col.size() : 1;
    CK(cudaMalloc(&op.rowptr, sizeof(int) * (P + 1)));
    CK(cudaMalloc(&op.col, sizeof(uint16_t) * nnz));
    CK(cudaMalloc(&op.val, sizeof(double2) * nnz));
    CK(cudaMalloc(&op.hdiag, sizeof(double2) * M));
    CK(cudaMalloc(&op.hfull, sizeof(double2) * M * M));
    CK(cudaMemcpyAsync(op.rowptr, rowptr.data(), sizeof(int) * (P + 1), cudaMemcpyHostToDevice, sp->stream));
    if (!col.empty()) {
        CK(cudaMemcpyAsync(op.col, col.data(), sizeof(uint16_t) * col.size(), cudaMemcpyHostToDevice, sp->stream));
        CK(cudaMemcpyAsync(op.val, val.data(), sizeof(double2) * val.size(), cudaMemcpyHostToDevice, sp->stream));
    }
    CK(cudaMemcpyAsync(op.hdiag, hdiag, sizeof(double2) * M, cudaMemcpyHostToDevice, sp->stream));
    CK(cudaMemcpyAsync(op.hfull, hfull, sizeof(double2) * M * M, cudaMemcpyHostToDevice, sp->stream));
    const std::vector<cplx> mom = pack_momentum(Ht, P, M);
    if (!mom.empty() && !sp->dense_only && sp->kernel_choice != 2) {
        CK(cudaMalloc(&op.hblk, sizeof(double2) * mom.size()));
        CK(cudaMemcpyAsync(op.hblk, mom.data(), sizeof(double2) * mom.size(), cudaMemcpyHostToDevice, sp->stream));
        op.nhblk = (int)mom.size();
        op.hblk_h.resize(mom.size());
        std::memcpy(op.hblk_h.data(), mom.data(), sizeof(double2) * mom.size());
    }
    const std::vector<int> prog = pack_blocks(Ht, P, M);
    if (!prog.empty() && !sp->dense_only) {
        CK(cudaMalloc(&op.prog, sizeof(int) * prog.size()));
        CK(cudaMemcpyAsync(op.prog, prog.data(), sizeof(int) * prog.size(), cudaMemcpyHostToDevice, sp->stream));
        op.prog_bytes = (int)(sizeof(int) * prog.size());
    }
    // General pair matrices: the register-tiled product does P^2 complex
    // multiply-adds per (N-2)-configuration at full FP64 rate, the CSR form
    // nnz at a fraction of it, so the dense form pays once a quarter is filled.
    const bool general = (mom.empty() || sp->kernel_choice == 2) && prog.empty() && 4 * col.size() >= (size_t)P * P;
    if (P <= mcpi::kGemmMaxP && !sp->no_gemm && (sp->dense_only || general)) {
        CK(cudaMalloc(&op.hdense, sizeof(double2) * P * P));
        CK(cudaMemcpyAsync(op.hdense, Ht.data(), sizeof(double2) * P * P, cudaMemcpyHostToDevice, sp->stream));
    }
    CK(cudaStreamSynchronize(sp->stream));  // host vectors go out of scope
    op.nnz = (int)col.size();
    return MCPI_OK;
}

// A grow-only device buffer of the space: reused when large enough, else replaced.
int reserve(void *&ptr, size_t &cap, size_t bytes)
{
    if (cap >= bytes && ptr) return MCPI_OK;
    cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    CK(cudaMalloc(&ptr, bytes ? bytes : 1));
    cap = bytes;
    return MCPI_OK;
}

int ensure_fused(mcpi_space_s *sp);

PairOp op_view(const mcpi_space_s *sp, const DevPairOp &op);

// The pair-space intermediate E (P x NC(N-2,M)) that the two-kernel and fused
// forms of op pass between their halves; the direct form needs none.
int ensure_E(mcpi_space_s *sp, const DevPairOp &op)
{
    if (sp->N < 2) return MCPI_OK;
    if (mcpi::hpsi_form(sp->sp, op_view(sp, op)) == mcpi::kFormDirect) return MCPI_OK;
    if (!sp->d_E) CK(cudaMalloc(&sp->d_E, sizeof(double2) * (size_t)sp->P * sp->nc2));
    return ensure_fused(sp);
}

void free_fused(mcpi_space_s *sp)
{
    if (sp->d_fz) {
        cudaStreamSynchronize(sp->stream);
        cudaFree(sp->d_fz);
    }
    sp->d_fz = nullptr;
    sp->fz = mcpi::FusedPlan{};
    sp->fz_ready = false;
}

// Builds the fused H.psi schedule of the space (FusedPlan, kernels.h): the
// highest producer tile each consumer tile reads, from the device, then the
// order -- before consumer tile c every producer tile up to need[c] + lead
// not yet listed, then c. Once per space (and after an option change).
int ensure_fused(mcpi_space_s *sp)
{
    if (!sp->fused_on || sp->fz_ready || sp->N < 2 || sp->M < 2) return MCPI_OK;
    const int64_t T = mcpi::kFusedTile;
    const int np = (int)((sp->nc2 + T - 1) / T), nct = (int)((sp->nc + T - 1) / T);
    const int ngroups = (np + mcpi::kFusedGroup - 1) / mcpi::kFusedGroup;
    // need | order | ctl (128-byte aligned) | count
    const size_t oc = ((size_t)nct + np + nct + 31) & ~size_t(31);
    const size_t words = oc + mcpi::kFusedCtlWords + ngroups;
    free_fused(sp);
    CK(cudaMalloc(&sp->d_fz, sizeof(int) * words));
    int *need = sp->d_fz, *order = need + nct;
    unsigned *ctl = (unsigned *)(sp->d_fz + oc), *count = ctl + mcpi::kFusedCtlWords;
    CK(cudaMemsetAsync(ctl, 0, sizeof(unsigned) * ((size_t)mcpi::kFusedCtlWords + ngroups), sp->stream));
    CK(mcpi::launch_fused_need(sp->sp, sp->tables(), need, sp->stream));
    std::vector<int> h_need(nct), h_order;
    h_order.reserve((size_t)np + nct);
    CK(cudaMemcpyAsync(h_need.data(), need, sizeof(int) * nct, cudaMemcpyDeviceToHost, sp->stream));
    CK(cudaStreamSynchronize(sp->stream));
    int next = 0;
    for (int c = 0; c < nct; ++c) {
        if (h_need[c] < 0 || h_need[c] >= np) return fail(MCPI_ERR_CUDA, "fused schedule: bad tile %d", h_need[c]);
        const int upto = std::min(np - 1, h_need[c] + sp->fused_lead);
        while (next <= upto) h_order.push_back(next++);
        h_order.push_back(-1 - c);
    }
    while (next < np) h_order.push_back(next++);
    CK(cudaMemcpyAsync(order, h_order.data(), sizeof(int) * h_order.size(), cudaMemcpyHostToDevice, sp->stream));
    int grid = 0;
    size_t smem = 0;
    CK(mcpi::fused_config(sp->sp, &grid, &smem));
    CK(cudaStreamSynchronize(sp->stream));   // h_order goes out of scope
    sp->fz.order = order;
    sp->fz.nitems = (int)h_order.size();
    sp->fz.need = need;
    sp->fz.count = count;
    sp->fz.ctl = ctl;
    sp->fz.np = np;
    sp->fz.grid = grid;
    sp->fz_ready = true;
    return MCPI_OK;
}

// The launch view of a pair operator, with the space's fused schedule
// attached when the fused form is on and built.
PairOp op_view(const mcpi_space_s *sp, const DevPairOp &op)
{
    PairOp v = op.view();
    if (sp->fused_on && sp->fz_ready) v.fused = sp->fz;
    v.direct = sp->direct_on;
    return v;
}

int ensure_gram(mcpi_space_s *sp)
{
    const size_t need = mcpi::gram_partial_elems(sp->sp, 2) > mcpi::gram_partial_elems(sp->sp, 1)
                            ? mcpi::gram_partial_elems(sp->sp, 2)
                            : mcpi::gram_partial_elems(sp->sp, 1);
    if (sp->gram_cap >= need) return MCPI_OK;
    cudaFree(sp->d_gram);
    sp->d_gram = nullptr;
    CK(cudaMalloc(&sp->d_gram, sizeof(double2) * need));
    sp->gram_cap = need;
    return MCPI_OK;
}

int apply_op(mcpi_space_s *sp, const DevPairOp &op, const void *d_C, void *d_out)
{
    CHECK_ARG(sp && d_C && d_out, "null argument");
    if (!sp->has_op) return fail(MCPI_ERR_STATE, "mcpi_set_integrals has not been called");
    CHECK_ARG(d_C != d_out, "input and output must not alias");
    DeviceGuard g(sp->device);
    int rc = ensure_E(sp, op);
    if (rc) return rc;
    CK(mcpi::launch_apply_h(sp->sp, sp->tables(), op_view(sp, op), op.blocks(), (const double2 *)d_C,
                            sp->d_E, (double2 *)d_out, sp->stream));
    return MCPI_OK;
}

}  // namespace

extern "C" {

static int check_status(mcpi_space_s *sp);

}  // extern "C"

int mcpi::set_error(int code, const char *msg)
{
    g_last_error = msg;
    return code;
}

extern "C" {

const char *mcpi_status_string(int status)
{
    switch (status) {
    case MCPI_OK: return "ok";
    case MCPI_ERR_ARG: return "invalid argument";
    case MCPI_ERR_RANGE: return "size out of supported range";
    case MCPI_ERR_CUDA: return "CUDA error";
    case MCPI_ERR_NOMEM: return "out of memory";
    case MCPI_ERR_STATE: return "invalid call order";
    case MCPI_ERR_NUMERIC: return "numerical failure";
    case MCPI_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
    }
}

const char *mcpi_last_error(void) { return g_last_error.c_str(); }

int mcpi_nc(int N, int M, int64_t *nc)
{
    CHECK_ARG(nc && N >= 0 && M >= 1, "mcpi_nc: need N >= 0, M >= 1");
    const int64_t v = nc_exact(N, M);
    if (v < 0) return fail(MCPI_ERR_RANGE, "NC(%d,%d) exceeds 63 bits", N, M);
    *nc = v;
    return MCPI_OK;
}

int mcpi_space_create(int N, int M, int device, mcpi_space *out)
{
    CHECK_ARG(out, "null output");
    *out = nullptr;
    CHECK_ARG(N >= 0 && M >= 1, "need N >= 0 and M >= 1");
    if (M > mcpi::kMaxM) return fail(MCPI_ERR_RANGE, "M=%d exceeds the supported %d orbitals", M, mcpi::kMaxM);
    const int64_t nc = nc_exact(N, M);
    if (nc < 0 || nc >= (int64_t)1 << 31)
        return fail(MCPI_ERR_RANGE, "NC(%d,%d) does not fit the 31-bit configuration index", N, M);
    const int ws = N + 3;
    if ((size_t)(M - 1) * ws * 4 + (size_t)ws * 8 > 24 * 1024)
        return fail(MCPI_ERR_RANGE, "N=%d too large for the shared-memory binomial table", N);
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    CHECK_ARG(device >= 0 && device < ndev, "invalid device ordinal");
    DeviceGuard g(device);
    auto *s = new mcpi_space_s;
    s->N = N;
    s->M = M;
    s->device = device;
    s->nc = nc;
    s->nc1 = N >= 1 ? nc_exact(N - 1, M) : 0;
    s->nc2 = N >= 2 ? nc_exact(N - 2, M) : 0;
    s->P = M * (M + 1) / 2;
    s->sp.N = N;
    s->sp.M = M;
    s->sp.wstride = ws;
    s->sp.nc = (uint32_t)nc;
    s->sp.nc1 = (uint32_t)s->nc1;
    s->sp.nc2 = (uint32_t)s->nc2;
    // W[i*ws + p] = C(p+i, i+1) mod 2^32, from Pascal's triangle mod 2^64 (exact modular)
    const int nmax = N + 2 + M;
    std::vector<std::vector<uint64_t>> C(nmax + 1, std::vector<uint64_t>(nmax + 1, 0));
    for (int n = 0; n <= nmax; ++n) {
        C[n][0] = 1;
        for (int k = 1; k <= n; ++k) C[n][k] = C[n - 1][k - 1] + (k <= n - 1 ? C[n - 1][k] : 0);
    }
    std::vector<uint32_t> W((size_t)(M > 1 ? M - 1 : 1) * ws, 0);
    for (int i = 0; i + 1 < M; ++i)
        for (int p = 0; p < ws; ++p) W[(size_t)i * ws + p] = (uint32_t)C[p + i][i + 1];
    std::vector<double> sq(ws);
    for (int n = 0; n < ws; ++n) sq[n] = std::sqrt((double)n);
    cudaError_t e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_W, sizeof(uint32_t) * W.size());
    if (e == cudaSuccess) e = cudaMalloc(&s->d_sq, sizeof(double) * ws);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_dot, sizeof(double2) * (mcpi::lanczos_parts(nc) + 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(s->d_status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(s->d_W, W.data(), sizeof(uint32_t) * W.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->d_sq, sq.data(), sizeof(double) * ws, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        mcpi_space_destroy(s);
        return fail(e == cudaErrorMemoryAllocation ? MCPI_ERR_NOMEM : MCPI_ERR_CUDA,
                    "mcpi_space_create: %s", cudaGetErrorString(e));
    }
    s->stream = s->own;
    *out = s;
    return MCPI_OK;
}

// Releases the host-buffer pipeline of mcpi_apply_h_host (whatever of it exists).
static void free_host_pipe(mcpi_space sp)
{
    if (sp->s_h2d) cudaStreamSynchronize(sp->s_h2d);
    if (sp->s_d2h) cudaStreamSynchronize(sp->s_d2h);
    for (int b = 0; b < 2; ++b) {
        cudaFree(sp->d_hin[b]);
        cudaFree(sp->d_hout[b]);
        if (sp->ev_in[b]) cudaEventDestroy(sp->ev_in[b]);
        if (sp->ev_comp[b]) cudaEventDestroy(sp->ev_comp[b]);
        if (sp->ev_out[b]) cudaEventDestroy(sp->ev_out[b]);
        sp->d_hin[b] = sp->d_hout[b] = nullptr;
        sp->ev_in[b] = sp->ev_comp[b] = sp->ev_out[b] = nullptr;
    }
    if (sp->s_h2d) cudaStreamDestroy(sp->s_h2d);
    if (sp->s_d2h) cudaStreamDestroy(sp->s_d2h);
    sp->s_h2d = sp->s_d2h = nullptr;
    sp->host_pipe_ready = false;
}

// Creates the pipeline: two streams, two input and two output buffers, and
// their events. On any failure everything created so far is released, so a
// later call starts again from nothing.
static cudaError_t make_host_pipe(mcpi_space sp, size_t bytes)
{
    cudaError_t e = cudaStreamCreateWithFlags(&sp->s_h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sp->s_d2h, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMalloc(&sp->d_hin[b], bytes);
        if (e == cudaSuccess) e = cudaMalloc(&sp->d_hout[b], bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sp->ev_in[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sp->ev_comp[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sp->ev_out[b], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        free_host_pipe(sp);
        return e;
    }
    sp->host_pipe_ready = true;
    return cudaSuccess;
}

int mcpi_space_destroy(mcpi_space sp)
{
    if (!sp) return MCPI_OK;
    DeviceGuard g(sp->device);
    if (sp->stream) cudaStreamSynchronize(sp->stream);
    free_op(sp->fwd);
    free_op(sp->adj);
    cudaFree(sp->d_W);
    cudaFree(sp->d_sq);
    cudaFree(sp->d_E);
    cudaFree(sp->d_gram);
    cudaFree(sp->d_dot);
    cudaFree(sp->d_status);
    cudaFree(sp->d_occ);
    cudaFree(sp->d_occ2);
    cudaFree(sp->d_occ1);
    cudaFree(sp->d_basis);
    cudaFree(sp->d_lzblk);
    cudaFree(sp->d_lzr);
    free_host_pipe(sp);
    free_fused(sp);
    cudaFree(sp->d_mr);
    if (sp->own) cudaStreamDestroy(sp->own);
    delete sp;
    return MCPI_OK;
}

int mcpi_space_set_stream(mcpi_space sp, void *stream)
{
    CHECK_ARG(sp, "null space");
    sp->stream = (cudaStream_t)stream;   // NULL selects the legacy default stream
    return MCPI_OK;
}

int mcpi_space_set_option(mcpi_space sp, int option, int value)
{
    CHECK_ARG(sp, "null space");
    switch (option) {
    case MCPI_OPT_DENSE_PAIR_KERNEL: sp->dense_only = value != 0; return MCPI_OK;
    case MCPI_OPT_NO_MOMENTUM_KERNEL: sp->kernel_choice = value ? 2 : 0; return MCPI_OK;
    case MCPI_OPT_NO_GEMM_KERNEL: sp->no_gemm = value != 0; return MCPI_OK;
    case MCPI_OPT_WAIT_LIMIT_KCYCLES:
        if (value < 0) return fail(MCPI_ERR_ARG, "wait limit must be >= 0");
        sp->wait_cycles = 1000LL * value;
        sp->fwd.wait_cycles = sp->adj.wait_cycles = sp->wait_cycles;
        return MCPI_OK;
    case MCPI_OPT_NO_OCC_TABLES:
        sp->no_occ = value != 0;
        if (sp->no_occ) {
            DeviceGuard g(sp->device);
            cudaStreamSynchronize(sp->stream);
            cudaFree(sp->d_occ);
            cudaFree(sp->d_occ2);
            cudaFree(sp->d_occ1);
            sp->d_occ = sp->d_occ2 = sp->d_occ1 = nullptr;
            sp->occ_bits = 0;
        }
        return MCPI_OK;
    case MCPI_OPT_TEST_STALL_GATHER:
        sp->test_stall = value != 0;
        sp->fwd.test_stall = sp->adj.test_stall = sp->test_stall;
        return MCPI_OK;
    case MCPI_OPT_FUSED_HPSI:
        if ((value != 0) != sp->fused_on) free_fused(sp);
        sp->fused_on = value != 0;
        return MCPI_OK;
    case MCPI_OPT_DIRECT_HPSI:
        if (value < 0) return fail(MCPI_ERR_ARG, "direct form must be >= 0");
        sp->direct_on = value;
        return MCPI_OK;
    case MCPI_OPT_FUSED_LEAD:
        if (value < 0) return fail(MCPI_ERR_ARG, "fused lead must be >= 0");
        if (value != sp->fused_lead) free_fused(sp);
        sp->fused_lead = value;
        return MCPI_OK;
    case MCPI_OPT_CREATE_FORM:
        sp->create_form = value;
        sp->fwd.create_form = sp->adj.create_form = value;
        return MCPI_OK;
    default: return fail(MCPI_ERR_ARG, "unknown option %d", option);
    }
}

// Reads and clears the device status word (after a stream synchronisation).
static int check_status(mcpi_space_s *sp)
{
    int st = 0;
    CK(cudaMemcpyAsync(&st, sp->d_status, sizeof(int), cudaMemcpyDeviceToHost, sp->stream));
    CK(cudaStreamSynchronize(sp->stream));
    if (st) {
        CK(cudaMemsetAsync(sp->d_status, 0, sizeof(int), sp->stream));
        return fail(MCPI_ERR_TIMEOUT, "a device-side bounded wait timed out (status %d)", st);
    }
    return MCPI_OK;
}

int mcpi_space_sync(mcpi_space sp)
{
    CHECK_ARG(sp, "null space");
    DeviceGuard g(sp->device);
    CK(cudaStreamSynchronize(sp->stream));
    return check_status(sp);
}

int mcpi_alloc(mcpi_space sp, size_t bytes, void **d_ptr)
{
    CHECK_ARG(sp && d_ptr, "null argument");
    DeviceGuard g(sp->device);
    *d_ptr = nullptr;
    CK(cudaMalloc(d_ptr, bytes ? bytes : 1));
    return MCPI_OK;
}

int mcpi_free(mcpi_space sp, void *d_ptr)
{
    CHECK_ARG(sp, "null space");
    DeviceGuard g(sp->device);
    CK(cudaFree(d_ptr));
    return MCPI_OK;
}

int mcpi_memcpy(mcpi_space sp, void *dst, const void *src, size_t bytes)
{
    CHECK_ARG(sp && (bytes == 0 || (dst && src)), "null argument");
    DeviceGuard g(sp->device);
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, sp->stream));
    CK(cudaStreamSynchronize(sp->stream));
    return check_status(sp);
}

int mcpi_space_dims(mcpi_space sp, int *N, int *M, int64_t *nc)
{
    CHECK_ARG(sp, "null space");
    if (N) *N = sp->N;
    if (M) *M = sp->M;
    if (nc) *nc = sp->nc;
    return MCPI_OK;
}

// ---- tables -----------------------------------------------------------------

int mcpi_ncmat(int N, int M, int32_t *h)
{
    CHECK_ARG(h && N >= 0 && M >= 1, "mcpi_ncmat: bad arguments");
    for (int n = 0; n <= N; ++n) {
        h[n] = 0;
        if (M >= 1) h[n + (N + 1)] = 1;
        for (int m = 2; m <= M; ++m) {
            const int64_t v = nc_exact(n, m);
            if (v < 0 || v > INT32_MAX) return fail(MCPI_ERR_RANGE, "NC(%d,%d) exceeds int32", n, m);
            h[n + (N + 1) * m] = (int32_t)v;
        }
    }
    return MCPI_OK;
}

int mcpi_index_to_fock(int N, int M, int64_t index, int32_t *v)
{
    CHECK_ARG(v && N >= 0 && M >= 1 && M <= 64, "mcpi_index_to_fock: bad arguments");
    const int64_t nc = nc_exact(N, M);
    CHECK_ARG(nc > 0 && index >= 0 && index < nc, "index out of range");
    // R = NC(N,M) - 1 - index = sum_i C(P_i + i, i+1); greedy from the top orbital
    unsigned __int128 R = (unsigned __int128)(nc - 1 - index);
    int hi = N;
    std::vector<int> P(M);
    P[M - 1] = N;
    for (int i = M - 2; i >= 0; --i) {
        int p = hi;
        while (p > 0 && binom128(p + i, i + 1) > R) --p;
        R -= binom128(p + i, i + 1);
        P[i] = p;
        hi = p;
    }
    v[0] = P[0];
    for (int i = 1; i < M; ++i) v[i] = P[i] - P[i - 1];
    return MCPI_OK;
}

int mcpi_fock_to_index(int N, int M, const int32_t *v, int64_t *index)
{
    CHECK_ARG(v && index && N >= 0 && M >= 1, "mcpi_fock_to_index: bad arguments");
    int64_t tot = 0;
    for (int i = 0; i < M; ++i) {
        CHECK_ARG(v[i] >= 0, "negative occupation");
        tot += v[i];
    }
    CHECK_ARG(tot == N, "occupations do not sum to N");
    unsigned __int128 s = 0;
    int64_t P = 0;
    for (int i = 0; i + 1 < M; ++i) {
        P += v[i];
        s += binom128(P + i, i + 1);
    }
    *index = nc_exact(N, M) - 1 - (int64_t)s;
    return MCPI_OK;
}

int mcpi_focks(mcpi_space sp, int32_t *d_IF)
{
    CHECK_ARG(sp && d_IF, "null argument");
    DeviceGuard g(sp->device);
    CK(mcpi::launch_focks(sp->sp, sp->tables(), d_IF, sp->stream));
    return MCPI_OK;
}

int mcpi_one_one_map(mcpi_space sp, int32_t *d_map)
{
    CHECK_ARG(sp && d_map, "null argument");
    DeviceGuard g(sp->device);
    CK(mcpi::launch_one_one_map(sp->sp, sp->tables(), d_map, sp->stream));
    return MCPI_OK;
}

int mcpi_two_map_size(mcpi_space sp, int two_orbital, int64_t *entries)
{
    CHECK_ARG(sp && entries, "null argument");
    DeviceGuard g(sp->device);
    int64_t *cnt = nullptr, *stride = nullptr, *tot = nullptr;
    void *scratch = nullptr;
    size_t need = 0;
    int rc = MCPI_OK;
    cudaError_t e = cudaMalloc(&cnt, sizeof(int64_t) * sp->nc);
    if (e == cudaSuccess) e = cudaMalloc(&stride, sizeof(int64_t) * sp->nc);
    if (e == cudaSuccess) e = cudaMalloc(&tot, sizeof(int64_t));
    if (e == cudaSuccess) e = mcpi::launch_chunk_counts(sp->sp, sp->tables(), two_orbital, cnt, sp->stream);
    if (e == cudaSuccess) e = mcpi::launch_stride_scan(sp->sp, cnt, stride, tot, nullptr, 0, &need, sp->stream);
    if (e == cudaSuccess) e = cudaMalloc(&scratch, need ? need : 1);
    if (e == cudaSuccess) e = mcpi::launch_stride_scan(sp->sp, cnt, stride, tot, scratch, need, nullptr, sp->stream);
    int64_t chunks = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&chunks, tot, sizeof(int64_t), cudaMemcpyDeviceToHost, sp->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sp->stream);
    if (e != cudaSuccess) rc = fail(MCPI_ERR_CUDA, "mcpi_two_map_size: %s", cudaGetErrorString(e));
    else *entries = chunks * sp->M * sp->M;
    cudaFree(cnt);
    cudaFree(stride);
    cudaFree(tot);
    cudaFree(scratch);
    return rc;
}

int mcpi_two_map(mcpi_space sp, int two_orbital, int64_t *d_stride, int32_t *d_map)
{
    CHECK_ARG(sp && d_stride && d_map, "null argument");
    DeviceGuard g(sp->device);
    int64_t *cnt = nullptr, *tot = nullptr;
    void *scratch = nullptr;
    size_t need = 0;
    int rc = MCPI_OK;
    cudaError_t e = cudaMalloc(&cnt, sizeof(int64_t) * sp->nc);
    if (e == cudaSuccess) e = cudaMalloc(&tot, sizeof(int64_t));
    if (e == cudaSuccess) e = mcpi::launch_chunk_counts(sp->sp, sp->tables(), two_orbital, cnt, sp->stream);
    if (e == cudaSuccess) e = mcpi::launch_stride_scan(sp->sp, cnt, d_stride, tot, nullptr, 0, &need, sp->stream);
    if (e == cudaSuccess) e = cudaMalloc(&scratch, need ? need : 1);
    if (e == cudaSuccess) e = mcpi::launch_stride_scan(sp->sp, cnt, d_stride, tot, scratch, need, nullptr, sp->stream);
    if (e == cudaSuccess) e = mcpi::launch_two_map(sp->sp, sp->tables(), two_orbital, d_stride, d_map, sp->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sp->stream);
    if (e != cudaSuccess) rc = fail(MCPI_ERR_CUDA, "mcpi_two_map: %s", cudaGetErrorString(e));
    cudaFree(cnt);
    cudaFree(tot);
    cudaFree(scratch);
    return rc;
}

// ---- operators -------------------------------------------------------------------

int mcpi_set_integrals(mcpi_space sp, const double *h_Ho, const double *h_Hint, int variant)
{
    CHECK_ARG(sp && h_Ho && h_Hint, "null argument");
    CHECK_ARG(variant == MCPI_VARIANT_MAPS || variant == MCPI_VARIANT_HASH, "unknown variant");
    DeviceGuard g(sp->device);
    const int M = sp->M, P = sp->P;
    const cplx *Ho = reinterpret_cast<const cplx *>(h_Ho);
    const cplx *Hint = reinterpret_cast<const cplx *>(h_Hint);
    std::vector<cplx> Ht = build_pair_matrix(sp->N, M, Ho, Hint, variant);
    std::vector<cplx> hd(M), hf(Ho, Ho + (size_t)M * M), hda(M), hfa((size_t)M * M);
    for (int k = 0; k < M; ++k) {
        hd[k] = Ho[k * M + k];
        hda[k] = std::conj(hd[k]);
        for (int l = 0; l < M; ++l) hfa[k * M + l] = std::conj(Ho[l * M + k]);
    }
    std::vector<cplx> Hta((size_t)P * P);
    for (int a = 0; a < P; ++a)
        for (int b = 0; b < P; ++b) Hta[(size_t)b * P + a] = std::conj(Ht[(size_t)a * P + b]);
    int rc = upload_op(sp, sp->fwd, Ht, hd.data(), hf.data());
    if (rc) return rc;
    rc = upload_op(sp, sp->adj, Hta, hda.data(), hfa.data());
    if (rc) return rc;
    sp->fwd.create_form = sp->adj.create_form = sp->create_form;
    sp->fwd.status = sp->adj.status = sp->d_status;
    sp->fwd.wait_cycles = sp->adj.wait_cycles = sp->wait_cycles;
    sp->fwd.test_stall = sp->adj.test_stall = sp->test_stall;
    // packed occupations of the N- and (N-2)-space rows, read by the H.psi
    // kernels instead of decoding each row index (8 bytes per configuration;
    // skipped, and the kernels decode, when they do not fit 64 bits or memory
    // is short)
    const int bits = mcpi::occ_bits_for(sp->N, sp->M);
    if (!sp->d_occ && !sp->no_occ && bits && sp->N >= 2 && sp->nc2 > 0) {
        const size_t b1 = sizeof(uint64_t) * (size_t)sp->nc, b2 = sizeof(uint64_t) * (size_t)sp->nc2;
        if (cudaMalloc(&sp->d_occ, b1) == cudaSuccess && cudaMalloc(&sp->d_occ2, b2) == cudaSuccess) {
            const mcpi::SpaceTables t{sp->d_W, sp->d_sq};
            mcpi::Space s2 = sp->sp;
            s2.N = sp->N - 2;
            s2.nc = (uint32_t)sp->nc2;
            CK(mcpi::launch_pack_occ(sp->sp, t, sp->d_occ, bits, sp->stream));
            CK(mcpi::launch_pack_occ(s2, t, sp->d_occ2, bits, sp->stream));
            sp->occ_bits = bits;
        } else {
            (void)cudaGetLastError();
            cudaFree(sp->d_occ);
            sp->d_occ = nullptr;
            sp->d_occ2 = nullptr;
        }
    }
    sp->has_op = true;
    return MCPI_OK;
}

int mcpi_apply_h(mcpi_space sp, const void *d_C, void *d_out) { return apply_op(sp, sp ? sp->fwd : DevPairOp{}, d_C, d_out); }

int mcpi_apply_h_host(mcpi_space sp, int count, const void *const *h_C, void *const *h_out)
{
    CHECK_ARG(sp && count >= 0 && (count == 0 || (h_C && h_out)), "mcpi_apply_h_host: bad arguments");
    if (!sp->has_op) return fail(MCPI_ERR_STATE, "mcpi_set_integrals has not been called");
    for (int k = 0; k < count; ++k) CHECK_ARG(h_C[k] && h_out[k], "mcpi_apply_h_host: null state pointer");
    DeviceGuard g(sp->device);
    int rc = ensure_E(sp, sp->fwd);
    if (rc) return rc;
    const size_t bytes = sizeof(double2) * (size_t)sp->nc;
    if (!sp->host_pipe_ready) CK(make_host_pipe(sp, bytes));
    // buffer pair b = k & 1: its input is free once H.psi of state k-2 has run,
    // its output once the copy out of state k-2 has finished
    for (int k = 0; k < count; ++k) {
        const int b = k & 1;
        if (k >= 2) CK(cudaStreamWaitEvent(sp->s_h2d, sp->ev_comp[b], 0));
        CK(cudaMemcpyAsync(sp->d_hin[b], h_C[k], bytes, cudaMemcpyHostToDevice, sp->s_h2d));
        CK(cudaEventRecord(sp->ev_in[b], sp->s_h2d));
        CK(cudaStreamWaitEvent(sp->stream, sp->ev_in[b], 0));
        if (k >= 2) CK(cudaStreamWaitEvent(sp->stream, sp->ev_out[b], 0));
        CK(mcpi::launch_apply_h(sp->sp, sp->tables(), op_view(sp, sp->fwd), sp->fwd.blocks(), sp->d_hin[b], sp->d_E,
                                sp->d_hout[b], sp->stream));
        CK(cudaEventRecord(sp->ev_comp[b], sp->stream));
        CK(cudaStreamWaitEvent(sp->s_d2h, sp->ev_comp[b], 0));
        CK(cudaMemcpyAsync(h_out[k], sp->d_hout[b], bytes, cudaMemcpyDeviceToHost, sp->s_d2h));
        CK(cudaEventRecord(sp->ev_out[b], sp->s_d2h));
    }
    CK(cudaStreamSynchronize(sp->s_d2h));
    CK(cudaStreamSynchronize(sp->stream));
    return check_status(sp);
}

int mcpi_apply_h_profile(mcpi_space sp, const void *d_C, void *d_out, int reps, float *h_ms)
{
    CHECK_ARG(sp && d_C && d_out && h_ms && reps >= 1, "mcpi_apply_h_profile: bad arguments");
    if (!sp->has_op) return fail(MCPI_ERR_STATE, "mcpi_set_integrals has not been called");
    DeviceGuard g(sp->device);
    int rc = ensure_E(sp, sp->fwd);
    if (rc) return rc;
    cudaEvent_t ev[3];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    float tot[2] = {0.f, 0.f};
    cudaError_t e = cudaSuccess;
    const PairOp fop = op_view(sp, sp->fwd);
    const bool one = mcpi::hpsi_form(sp->sp, fop) != mcpi::kFormTwo;
    if (one) {
        // direct or fused form: one kernel, reported as h_ms[0]
        for (int r = 0; r < reps && e == cudaSuccess; ++r) {
            e = cudaEventRecord(ev[0], sp->stream);
            if (e == cudaSuccess)
                e = mcpi::launch_apply_h(sp->sp, sp->tables(), fop, sp->fwd.blocks(), (const double2 *)d_C,
                                         sp->d_E, (double2 *)d_out, sp->stream, 3);
            if (e == cudaSuccess) e = cudaEventRecord(ev[1], sp->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
            float a = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&a, ev[0], ev[1]);
            tot[0] += a;
        }
    }
    for (int r = 0; r < reps && e == cudaSuccess && !one; ++r) {
        e = cudaEventRecord(ev[0], sp->stream);
        if (e == cudaSuccess)
            e = mcpi::launch_apply_h(sp->sp, sp->tables(), sp->fwd.view(), sp->fwd.blocks(),
                                     (const double2 *)d_C, sp->d_E, (double2 *)d_out, sp->stream, 1);
        if (e == cudaSuccess) e = cudaEventRecord(ev[1], sp->stream);
        if (e == cudaSuccess)
            e = mcpi::launch_apply_h(sp->sp, sp->tables(), sp->fwd.view(), sp->fwd.blocks(),
                                     (const double2 *)d_C, sp->d_E, (double2 *)d_out, sp->stream, 2);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2], sp->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[2]);
        float a = 0.f, b = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&a, ev[0], ev[1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&b, ev[1], ev[2]);
        tot[0] += a;
        tot[1] += b;
    }
    for (auto &x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) return fail(MCPI_ERR_CUDA, "mcpi_apply_h_profile: %s", cudaGetErrorString(e));
    h_ms[0] = tot[0] / reps;
    h_ms[1] = tot[1] / reps;
    return MCPI_OK;
}

int mcpi_apply_h_rows(mcpi_space sp, const void *d_C, int64_t row0, int64_t row1, void *d_out)
{
    CHECK_ARG(sp && d_C && d_C != d_out, "mcpi_apply_h_rows: bad arguments");
    CHECK_ARG(row0 >= 0 && row0 <= row1 && row1 <= sp->nc, "mcpi_apply_h_rows: bad row range");
    if (row0 == row1) return MCPI_OK;
    CHECK_ARG(d_out, "mcpi_apply_h_rows: null output");
    if (!sp->has_op) return fail(MCPI_ERR_STATE, "mcpi_set_integrals has not been called");
    if (sp->N < 2 || sp->create_form != 0)
        return fail(MCPI_ERR_ARG, "row ranges need N >= 2 and the default pair-creation form");
    DeviceGuard g(sp->device);
    int rc = ensure_E(sp, sp->fwd);
    if (rc) return rc;
    // kernel 1 only over the E columns these rows read (momentum-block form):
    // a rank of a sharded solve does not recompute the whole intermediate.
    // The range is found once per row block (one pass over its rows).
    uint32_t m0 = 0, m1 = 0xffffffffu;
    const PairOp fop = op_view(sp, sp->fwd);
    if (sp->fwd.hblk && sp->M >= 2 && mcpi::hpsi_form(sp->sp, fop) != mcpi::kFormDirect) {
        if (sp->mr_r0 != row0 || sp->mr_r1 != row1) {
            if (!sp->d_mr) CK(cudaMalloc(&sp->d_mr, 2 * sizeof(uint32_t)));
            uint32_t h[2];
            CK(mcpi::launch_rows_mrange(sp->sp, sp->tables(), (uint32_t)row0, (uint32_t)row1, sp->d_mr, sp->stream));
            CK(cudaMemcpyAsync(h, sp->d_mr, sizeof h, cudaMemcpyDeviceToHost, sp->stream));
            CK(cudaStreamSynchronize(sp->stream));
            if (h[0] > h[1] || h[1] >= sp->nc2) return fail(MCPI_ERR_CUDA, "row block range: bad columns");
            sp->mr_r0 = row0;
            sp->mr_r1 = row1;
            sp->mr_lo = h[0];
            sp->mr_hi = h[1];
        }
        m0 = sp->mr_lo;
        m1 = sp->mr_hi + 1;
    }
    CK(mcpi::launch_apply_h(sp->sp, sp->tables(), fop, sp->fwd.blocks(), (const double2 *)d_C,
                            sp->d_E, (double2 *)d_out, sp->stream, 3, (uint32_t)row0, (uint32_t)row1, m0, m1));
    return MCPI_OK;
}

int mcpi_apply_h_adjoint(mcpi_space sp, const void *d_C, void *d_out)
{
    return apply_op(sp, sp ? sp->adj : DevPairOp{}, d_C, d_out);
}

static int density(mcpi_space sp, int order, const void *phi, const void *psi, void *out)
{
    CHECK_ARG(sp && phi && psi && out, "null argument");
    DeviceGuard g(sp->device);
    int rc = ensure_gram(sp);
    if (rc) return rc;
    // rho1 reads the packed occupations of the (N-1)-space, built on its first
    // call with the bits of the space's other tables (none: the kernel decodes)
    if (order == 1 && !sp->d_occ1 && sp->occ_bits && sp->nc1 > 0) {
        if (cudaMalloc(&sp->d_occ1, sizeof(uint64_t) * (size_t)sp->nc1) == cudaSuccess) {
            mcpi::Space s1 = sp->sp;
            s1.N = sp->N - 1;
            s1.nc = (uint32_t)sp->nc1;
            CK(mcpi::launch_pack_occ(s1, mcpi::SpaceTables{sp->d_W, sp->d_sq}, sp->d_occ1, sp->occ_bits,
                                     sp->stream));
        } else {
            (void)cudaGetLastError();
            sp->d_occ1 = nullptr;
        }
    }
    CK(mcpi::launch_density(sp->sp, sp->tables(), order, (const double2 *)phi, (const double2 *)psi,
                            sp->d_gram, (double2 *)out, sp->stream, sp->d_status, sp->wait_cycles,
                            sp->test_stall));
    return MCPI_OK;
}

int mcpi_rho1(mcpi_space sp, const void *d_C, void *d_rho1) { return density(sp, 1, d_C, d_C, d_rho1); }
int mcpi_rho2(mcpi_space sp, const void *d_C, void *d_rho2) { return density(sp, 2, d_C, d_C, d_rho2); }
int mcpi_trans_rho1(mcpi_space sp, const void *phi, const void *psi, void *t1) { return density(sp, 1, phi, psi, t1); }
int mcpi_trans_rho2(mcpi_space sp, const void *phi, const void *psi, void *t2) { return density(sp, 2, phi, psi, t2); }

// ---- row-shard Lanczos primitives ------------------------------------------------------

#define SHARD_CK(call)                                                                      \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess) return fail(MCPI_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
    } while (0)

size_t mcpi_shard_scratch_elems(int64_t n, int lm) { return n < 0 || lm < 1 ? 0 : mcpi::shard_scratch_elems(n, lm); }

int mcpi_shard_scale(int64_t n, const void *d_r, void *d_vnext, const double *d_beta_i, const int *d_done,
                     void *stream)
{
    CHECK_ARG(n >= 0 && d_r && d_vnext && d_beta_i && d_done, "mcpi_shard_scale: bad arguments");
    if (n == 0) return MCPI_OK;
    SHARD_CK(mcpi::launch_shard_scale(n, (const double2 *)d_r, (double2 *)d_vnext, d_beta_i, d_done,
                                      (cudaStream_t)stream));
    return MCPI_OK;
}

int mcpi_shard_axpy_dot(int64_t n, const void *d_vprev, const void *d_vcur, void *d_r, const double *d_beta_i,
                        void *d_scratch, void *d_dot, const int *d_done, void *stream)
{
    CHECK_ARG(n >= 0 && d_vcur && d_r && d_scratch && d_dot && d_done && (!d_vprev || d_beta_i),
              "mcpi_shard_axpy_dot: bad arguments");
    SHARD_CK(mcpi::launch_shard_axpy_dot(n, (const double2 *)d_vprev, (const double2 *)d_vcur, (double2 *)d_r,
                                         d_beta_i, (double2 *)d_scratch, (double2 *)d_dot, d_done,
                                         (cudaStream_t)stream));
    return MCPI_OK;
}

int mcpi_shard_multidot(int64_t n, const void *d_V, int nvec, const void *d_r, const void *d_vcur,
                        const void *d_alpha, void *d_scratch, void *d_coef, const int *d_done, void *stream)
{
    CHECK_ARG(n >= 0 && nvec >= 1 && d_V && d_r && d_vcur && d_alpha && d_scratch && d_coef && d_done,
              "mcpi_shard_multidot: bad arguments");
    SHARD_CK(mcpi::launch_shard_multidot(n, (const double2 *)d_V, nvec, (const double2 *)d_r,
                                         (const double2 *)d_vcur, (const double2 *)d_alpha, (double2 *)d_scratch,
                                         (double2 *)d_coef, d_done, (cudaStream_t)stream));
    return MCPI_OK;
}

int mcpi_shard_update(int64_t n, const void *d_V, int nvec, void *d_r, const void *d_vcur, const void *d_alpha,
                      const void *d_coef, void *d_scratch, double *d_norm2, const int *d_done, void *stream)
{
    CHECK_ARG(n >= 0 && nvec >= 0 && (nvec == 0 || (d_V && d_coef)) && d_r && d_vcur && d_alpha && d_scratch &&
                  d_norm2 && d_done,
              "mcpi_shard_update: bad arguments");
    SHARD_CK(mcpi::launch_shard_update(n, (const double2 *)d_V, nvec, (double2 *)d_r, (const double2 *)d_vcur,
                                       (const double2 *)d_alpha, (const double2 *)d_coef, (double2 *)d_scratch,
                                       d_norm2, d_done, (cudaStream_t)stream));
    return MCPI_OK;
}

int mcpi_shard_beta(int i, double tol, const double *d_norm2, double *d_beta, double *d_maxbeta, int *d_done,
                    int *d_iters, void *stream)
{
    CHECK_ARG(i >= 0 && d_norm2 && d_beta && d_maxbeta && d_done && d_iters, "mcpi_shard_beta: bad arguments");
    SHARD_CK(mcpi::launch_shard_beta(i, tol, d_norm2, d_beta, d_maxbeta, d_done, d_iters, (cudaStream_t)stream));
    return MCPI_OK;
}

int mcpi_shard_combine(int64_t n, const void *d_V, int nvec, const double *d_z, void *d_out, void *stream)
{
    CHECK_ARG(n >= 0 && nvec >= 1 && d_V && d_z && d_out, "mcpi_shard_combine: bad arguments");
    if (n == 0) return MCPI_OK;
    SHARD_CK(mcpi::launch_combine((const double2 *)d_V, nvec, n, d_z, (double2 *)d_out, (cudaStream_t)stream));
    return MCPI_OK;
}

int mcpi_dot(mcpi_space sp, const void *d_a, const void *d_b, double *h_result2)
{
    CHECK_ARG(sp && d_a && d_b && h_result2, "null argument");
    DeviceGuard g(sp->device);
    CK(mcpi::launch_dot((const double2 *)d_a, (const double2 *)d_b, sp->nc, sp->d_dot + 1, sp->d_dot,
                        sp->stream));
    CK(cudaMemcpyAsync(h_result2, sp->d_dot, sizeof(double2), cudaMemcpyDeviceToHost, sp->stream));
    CK(cudaStreamSynchronize(sp->stream));
    return MCPI_OK;
}

// ---- Lanczos -------------------------------------------------------------------------

int mcpi_lanczos(mcpi_space sp, void *d_lvec, int lm, double *h_diag, double *h_offdiag, int *iters)
{
    CHECK_ARG(sp && d_lvec && lm >= 1, "mcpi_lanczos: bad arguments");
    if (!sp->has_op) return fail(MCPI_ERR_STATE, "mcpi_set_integrals has not been called");
    DeviceGuard g(sp->device);
    int rc = ensure_E(sp, sp->fwd);
    if (rc) return rc;
    const int64_t nc = sp->nc;
    const size_t npart = mcpi::lanczos_partial_elems(nc, lm);
    // state block: alpha(lm) coef(lm) partial(npart) | beta(lm) maxbeta | done iters
    const size_t bytes = sizeof(double2) * (2 * (size_t)lm + npart) + sizeof(double) * (lm + 1) + 2 * sizeof(int);
    rc = reserve(sp->d_lzblk, sp->lzblk_cap, bytes);
    if (rc) return rc;
    rc = reserve(sp->d_lzr, sp->lzr_cap, sizeof(double2) * nc);
    if (rc) return rc;
    char *blk = (char *)sp->d_lzblk;
    double2 *r = (double2 *)sp->d_lzr;
    cudaError_t e = cudaSuccess;
    mcpi::LanczosState s;
    s.alpha = (double2 *)blk;
    s.coef = s.alpha + lm;
    s.partial = s.coef + lm;
    s.beta = (double *)(s.partial + npart);
    s.maxbeta = s.beta + lm;
    s.done = (int *)(s.maxbeta + 1);
    s.iters = s.done + 1;
    s.nparts = mcpi::lanczos_parts(nc);
    const int init[2] = {0, lm};
    double2 *V = (double2 *)d_lvec;
    const PairOp op = op_view(sp, sp->fwd);
    const mcpi::BlockOp bo = sp->fwd.blocks();
    const SpaceTables tb = sp->tables();
    e = cudaMemsetAsync(blk, 0, bytes, sp->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.done, init, sizeof init, cudaMemcpyHostToDevice, sp->stream);
    if (e == cudaSuccess) e = mcpi::launch_apply_h(sp->sp, tb, op, bo, V, sp->d_E, r, sp->stream);
    if (e == cudaSuccess) e = mcpi::launch_lanczos_start(V, r, r, nc, s, sp->stream);
    for (int i = 0; i < lm - 1 && e == cudaSuccess; ++i) {
        double2 *vi = V + (size_t)i * nc, *vn = V + (size_t)(i + 1) * nc;
        e = mcpi::launch_lanczos_beta(i, lm, 1e-15, s, sp->stream);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_scale(r, vn, nc, i, s, sp->stream);
        if (e == cudaSuccess) e = mcpi::launch_apply_h(sp->sp, tb, op, bo, vn, sp->d_E, r, sp->stream);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_alpha(vi, vn, r, nc, i, s, sp->stream);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_reorth(V, i + 2, r, nc, i, s, sp->stream);
    }
    std::vector<double2> alpha(lm);
    std::vector<double> beta(lm);
    int it = lm;
    if (e == cudaSuccess) e = cudaMemcpyAsync(alpha.data(), s.alpha, sizeof(double2) * lm, cudaMemcpyDeviceToHost, sp->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(beta.data(), s.beta, sizeof(double) * lm, cudaMemcpyDeviceToHost, sp->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&it, s.iters, sizeof(int), cudaMemcpyDeviceToHost, sp->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sp->stream);
    if (e != cudaSuccess) return fail(MCPI_ERR_CUDA, "mcpi_lanczos: %s", cudaGetErrorString(e));
    rc = check_status(sp);
    if (rc) return rc;
    if (h_diag) std::memcpy(h_diag, alpha.data(), sizeof(double2) * lm);
    if (h_offdiag) {
        for (int i = 0; i < lm; ++i) h_offdiag[i] = i < lm - 1 ? beta[i] : 0.0;
    }
    if (iters) *iters = it;
    return MCPI_OK;
}

int mcpi_tridiag_eig(int n, double *d, double *e, double *z)
{
    CHECK_ARG(n >= 0 && (n == 0 || (d && (n == 1 || e))), "mcpi_tridiag_eig: bad arguments");
    if (mcpi::tridiag_eig(n, d, e, z) != 0) return fail(MCPI_ERR_NUMERIC, "tridiagonal QL did not converge");
    return MCPI_OK;
}

int mcpi_ground(mcpi_space sp, void *d_C, int niter, double *E0, int *iters)
{
    CHECK_ARG(sp && d_C && E0 && niter >= 1, "mcpi_ground: bad arguments");
    DeviceGuard g(sp->device);
    const int64_t nc = sp->nc;
    int rc0 = reserve(sp->d_basis, sp->basis_cap, sizeof(double2) * nc * (size_t)niter);
    if (rc0) return rc0;
    double2 *V = (double2 *)sp->d_basis;
    cudaError_t e = cudaMemcpyAsync(V, d_C, sizeof(double2) * nc, cudaMemcpyDeviceToDevice, sp->stream);
    if (e != cudaSuccess) return fail(MCPI_ERR_CUDA, "mcpi_ground: %s", cudaGetErrorString(e));
    std::vector<double> diag(2 * (size_t)niter), off(niter);
    int it = 0;
    int rc = mcpi_lanczos(sp, V, niter, diag.data(), off.data(), &it);
    if (rc) return rc;
    // groundStateLieb.c:419-449; a breakdown at the first step keeps alpha_0
    const int n = it > 0 ? it : 1;
    std::vector<double> d(n), ee(n > 1 ? n - 1 : 1), z((size_t)n * n);
    for (int k = 0; k < n; ++k) d[k] = diag[2 * k];
    for (int k = 0; k + 1 < n; ++k) ee[k] = off[k];
    if (mcpi::tridiag_eig(n, d.data(), ee.data(), z.data()) != 0)
        return fail(MCPI_ERR_NUMERIC, "tridiagonal QL did not converge");
    double sentinel = 1e10;
    int jmin = 0;
    for (int k = 0; k < n; ++k)
        if (sentinel > d[k]) {
            sentinel = d[k];
            jmin = k;
        }
    std::vector<double> zc(n);
    for (int k = 0; k < n; ++k) zc[k] = z[(size_t)k * n + jmin];
    double *dz = nullptr;
    e = cudaMalloc(&dz, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dz, zc.data(), sizeof(double) * n, cudaMemcpyHostToDevice, sp->stream);
    if (e == cudaSuccess) e = mcpi::launch_combine(V, n, nc, dz, (double2 *)d_C, sp->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sp->stream);
    cudaFree(dz);
    if (e != cudaSuccess) return fail(MCPI_ERR_CUDA, "mcpi_ground: %s", cudaGetErrorString(e));
    *E0 = d[jmin];
    if (iters) *iters = it;
    return MCPI_OK;
}

// Two-pass Lanczos without reorthogonalisation, for spaces whose Krylov basis
// does not fit: pass 1 keeps three vectors and records alpha/beta; pass 2
// regenerates the same Krylov vectors from the stored alpha/beta (every kernel
// and reduction is deterministic, so they are bitwise those of pass 1) and
// accumulates the Ritz vector. Same breakdown rule as mcpi_lanczos.
int mcpi_ground_lowmem(mcpi_space sp, void *d_C, int niter, double *E0, int *iters)
{
    CHECK_ARG(sp && d_C && E0 && niter >= 1 && niter <= 1 << 20, "mcpi_ground_lowmem: bad arguments");
    if (!sp->has_op) return fail(MCPI_ERR_STATE, "mcpi_set_integrals has not been called");
    DeviceGuard g(sp->device);
    int rc = ensure_E(sp, sp->fwd);
    if (rc) return rc;
    const int64_t nc = sp->nc;
    const int lm = niter;
    const size_t npart = mcpi::lanczos_partial_elems(nc, 1);
    // state: alpha(lm) coef(lm) partial(npart) | beta(lm) maxbeta z(lm) | done iters
    const size_t sbytes = sizeof(double2) * (2 * (size_t)lm + npart) + sizeof(double) * (2 * (size_t)lm + 1) +
                          2 * sizeof(int);
    char *blk = nullptr;
    double2 *vec = nullptr;   // v[0], v[1], r, acc
    CK(cudaMalloc(&blk, sbytes));
    cudaError_t e = cudaMalloc(&vec, sizeof(double2) * nc * 4);
    if (e != cudaSuccess) {
        cudaFree(blk);
        return fail(MCPI_ERR_NOMEM, "mcpi_ground_lowmem: %s", cudaGetErrorString(e));
    }
    mcpi::LanczosState s;
    s.alpha = (double2 *)blk;
    s.coef = s.alpha + lm;
    s.partial = s.coef + lm;
    s.beta = (double *)(s.partial + npart);
    s.maxbeta = s.beta + lm;
    double *dz = s.maxbeta + 1;
    s.done = (int *)(dz + lm);
    s.iters = s.done + 1;
    s.nparts = mcpi::lanczos_parts(nc);
    double2 *v[2] = {vec, vec + nc}, *r = vec + 2 * nc, *acc = vec + 3 * nc;
    const PairOp op = op_view(sp, sp->fwd);
    const mcpi::BlockOp bo = sp->fwd.blocks();
    const SpaceTables tb = sp->tables();
    const int init[2] = {0, lm};
    cudaStream_t st = sp->stream;
    // pass 1: tridiagonal only
    e = cudaMemsetAsync(blk, 0, sbytes, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.done, init, sizeof init, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v[0], d_C, sizeof(double2) * nc, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = mcpi::launch_apply_h(sp->sp, tb, op, bo, v[0], sp->d_E, r, st);
    if (e == cudaSuccess) e = mcpi::launch_lanczos_start(v[0], r, r, nc, s, st);
    for (int i = 0; i < lm - 1 && e == cudaSuccess; ++i) {
        double2 *vi = v[i & 1], *vn = v[(i + 1) & 1];
        e = mcpi::launch_lanczos_beta(i, lm, 1e-15, s, st);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_scale(r, vn, nc, i, s, st);
        if (e == cudaSuccess) e = mcpi::launch_apply_h(sp->sp, tb, op, bo, vn, sp->d_E, r, st);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_alpha(vi, vn, r, nc, i, s, st);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_no_reorth(vn, r, nc, i, s, st);
    }
    std::vector<double2> alpha(lm);
    std::vector<double> beta(lm);
    int it = lm;
    if (e == cudaSuccess) e = cudaMemcpyAsync(alpha.data(), s.alpha, sizeof(double2) * lm, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(beta.data(), s.beta, sizeof(double) * lm, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&it, s.iters, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    const int n = it > 0 ? it : 1;
    std::vector<double> d(n), ee(n > 1 ? n - 1 : 1), z((size_t)n * n), zc(lm, 0.0);
    int jmin = 0;
    if (e == cudaSuccess) {
        for (int k = 0; k < n; ++k) d[k] = alpha[k].x;
        for (int k = 0; k + 1 < n; ++k) ee[k] = beta[k];
        if (mcpi::tridiag_eig(n, d.data(), ee.data(), z.data()) != 0) {
            cudaFree(blk);
            cudaFree(vec);
            return fail(MCPI_ERR_NUMERIC, "tridiagonal QL did not converge");
        }
        double sentinel = 1e10;
        for (int k = 0; k < n; ++k)
            if (sentinel > d[k]) {
                sentinel = d[k];
                jmin = k;
            }
        for (int k = 0; k < n; ++k) zc[k] = z[(size_t)k * n + jmin];
    }
    // pass 2: regenerate v_0 .. v_{n-1} and accumulate sum_k z_k v_k
    if (e == cudaSuccess) e = cudaMemcpyAsync(dz, zc.data(), sizeof(double) * lm, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.done, init, sizeof init, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v[0], d_C, sizeof(double2) * nc, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = mcpi::launch_apply_h(sp->sp, tb, op, bo, v[0], sp->d_E, r, st);
    if (e == cudaSuccess) e = mcpi::launch_lanczos_no_reorth(v[0], r, nc, -1, s, st);
    if (e == cudaSuccess) e = mcpi::launch_axpy_real(acc, v[0], nc, dz, 1, st);
    for (int i = 0; i < n - 1 && e == cudaSuccess; ++i) {
        double2 *vi = v[i & 1], *vn = v[(i + 1) & 1];
        e = mcpi::launch_lanczos_scale(r, vn, nc, i, s, st);
        if (e == cudaSuccess) e = mcpi::launch_apply_h(sp->sp, tb, op, bo, vn, sp->d_E, r, st);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_axpy(vi, r, nc, i, s, st);
        if (e == cudaSuccess) e = mcpi::launch_lanczos_no_reorth(vn, r, nc, i, s, st);
        if (e == cudaSuccess) e = mcpi::launch_axpy_real(acc, vn, nc, dz + i + 1, 0, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_C, acc, sizeof(double2) * nc, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(blk);
    cudaFree(vec);
    if (e != cudaSuccess) return fail(MCPI_ERR_CUDA, "mcpi_ground_lowmem: %s", cudaGetErrorString(e));
    *E0 = d[jmin];
    if (iters) *iters = it;
    return check_status(sp);
}

int mcpi_lieb_integrals(int M, double g, double L, double *h_Ho, double *h_Hint)
{
    CHECK_ARG(M >= 1 && h_Ho && h_Hint && L > 0, "mcpi_lieb_integrals: bad arguments");
    const double pi = 3.141592653589793;
    cplx *Ho = reinterpret_cast<cplx *>(h_Ho);
    cplx *Hint = reinterpret_cast<cplx *>(h_Hint);
    for (int n = 0; n < M; ++n) {
        const double k = 2 * pi * (n - M / 2) / L;
        for (int j = 0; j < M; ++j) Ho[n * M + j] = 0.0;
        Ho[n * M + n] = 0.5 * k * k;
    }
    const size_t M2 = (size_t)M * M, M3 = M2 * M;
    for (int n = 0; n < M; ++n)
        for (int s = 0; s < M; ++s)
            for (int q = 0; q < M; ++q)
                for (int l = 0; l < M; ++l)
                    Hint[n + s * M + q * M2 + l * M3] = (l + q - s - n == 0) ? g : 0.0;
    return MCPI_OK;
}

}  // extern "C"
