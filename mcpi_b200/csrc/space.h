// Internal definition of the space context shared by the host-side
// translation units (capi.cpp, batch.cu). Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/mcpi_b200.h"
#include "kernels.h"

namespace mcpi {

struct DevPairOp {
    int *rowptr = nullptr;
    uint16_t *col = nullptr;
    double2 *val = nullptr;
    double2 *hdiag = nullptr;
    double2 *hfull = nullptr;
    int nnz = 0;
    int *prog = nullptr;       // block-sparse form (nullptr when a block is too wide)
    int prog_bytes = 0;
    double2 *hblk = nullptr;   // momentum-block form (nullptr when Ht couples different q+l)
    int nhblk = 0;
    std::vector<double2> hblk_h;   // host copy of hblk
    int create_form = 0;
    int *status = nullptr;     // the space's device status word (not owned)
    double2 *hdense = nullptr; // dense form (nullptr unless Ht is general and P <= kGemmMaxP)
    long long wait_cycles = 0;
    int test_stall = 0;
    PairOp view() const
    {
        return PairOp{rowptr, col, val, hdiag, hfull, nnz, hblk, nhblk, create_form, status, hdense,
                      wait_cycles, test_stall, hblk_h.empty() ? nullptr : hblk_h.data(), FusedPlan{}, 0};
    }
    BlockOp blocks() const { return BlockOp{prog, prog_bytes}; }
};

// Records msg as the calling thread's mcpi_last_error() and returns code.
int set_error(int code, const char *msg);

}  // namespace mcpi

struct mcpi_space_s {
    int N = 0, M = 0, device = 0;
    mcpi::Space sp{};
    int64_t nc = 0, nc1 = 0, nc2 = 0;
    int P = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    // host-buffer pipeline of mcpi_apply_h_host (created at its first call)
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
    double2 *d_hin[2] = {nullptr, nullptr}, *d_hout[2] = {nullptr, nullptr};
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
    bool host_pipe_ready = false;    // set only once every resource above exists
    uint32_t *d_W = nullptr;
    double *d_sq = nullptr;
    bool has_op = false;
    mcpi::DevPairOp fwd, adj;
    double2 *d_E = nullptr;          // P * nc2 scratch of H.psi
    double2 *d_gram = nullptr;       // density partials
    size_t gram_cap = 0;
    double2 *d_dot = nullptr;        // 1 result + partials
    int *d_status = nullptr;         // device status word: 1 = a kernel's bounded wait timed out
    bool dense_only = false;         // force the dense pair-matrix kernel
    int kernel_choice = 0;           // 2: skip the momentum-block kernel
    bool no_gemm = false;            // general pair matrices use the CSR kernel (MCPI_OPT_NO_GEMM_KERNEL)
    long long wait_cycles = 0;       // MCPI_OPT_WAIT_LIMIT_CYCLES
    int test_stall = 0;              // MCPI_OPT_TEST_STALL_GATHER
    bool no_occ = false;             // MCPI_OPT_NO_OCC_TABLES
    int create_form = 0;            // pair-creation kernel form (MCPI_OPT_CREATE_FORM)
    // fused H.psi (MCPI_OPT_FUSED_*): schedule built once per space by ensure_fused
    bool fused_on = false;
    int direct_on = 2;               // MCPI_OPT_DIRECT_HPSI (default: on for M <= 11)
    int fused_lead = 128;
    bool fz_ready = false;
    mcpi::FusedPlan fz{};
    int *d_fz = nullptr;             // one allocation: need | order | ctl | count
    // mcpi_apply_h_rows: the (N-2)-configuration range its last row block reads
    int64_t mr_r0 = -1, mr_r1 = -1;
    uint32_t mr_lo = 0, mr_hi = 0;
    uint32_t *d_mr = nullptr;
    // grow-only workspaces kept between calls: Krylov basis of mcpi_ground,
    // state block and residual of mcpi_lanczos
    void *d_basis = nullptr, *d_lzblk = nullptr, *d_lzr = nullptr;
    size_t basis_cap = 0, lzblk_cap = 0, lzr_cap = 0;
    uint64_t *d_occ = nullptr;       // packed occupations of the space's rows (built by mcpi_set_integrals)
    uint64_t *d_occ2 = nullptr;      // the same for the (N-2)-particle space
    uint64_t *d_occ1 = nullptr;      // the same for the (N-1)-particle space (first rho1 call)
    int occ_bits = 0;
    mcpi::SpaceTables tables() const { return mcpi::SpaceTables{d_W, d_sq, d_occ, occ_bits, d_occ2, d_occ1}; }
};
