// Internal launch interface between the C ABI layer (capi.cpp) and the CUDA
// translation units. Nothing here is part of the public ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fock.cuh"

namespace mcpi {

// Fused H.psi (momentum-block form only). One persistent launch runs the
// tiles of kernel 1 (producers: 256 (N-2)-configurations each, writing E) and
// of kernel 2 (consumers: 256 rows each, reading E) in one interleaved order,
// so that E is read back while it is still in L2 instead of making a round
// trip through HBM. Blocks take items in that order from a ticket counter; a
// consumer waits (bounded) until every producer tile up to need[c] has
// counted itself done. Built once per space (capi.cpp: ensure_fused).
constexpr int kFusedTile = 256;      // configurations per producer tile = rows per consumer tile
constexpr int kFusedGroup = 16;      // producer tiles per completion counter
constexpr int kFusedCtlWords = 96;   // ticket, exited, abort: one 128-byte line each
struct FusedPlan {
    const int *order = nullptr;  // nitems: producer tile p >= 0, or -1 - c for consumer tile c
    int nitems = 0;
    const int *need = nullptr;   // per consumer tile: the highest producer tile it reads
    unsigned *count = nullptr;   // per group of kFusedGroup producer tiles: tiles done (zero between calls)
    unsigned *ctl = nullptr;     // control words (zero between calls)
    int np = 0;                  // producer tiles
    int grid = 0;                // persistent blocks
};

// Two-body operator in pair form: H2 = sum_{a,b} Ht[a][b] A+_a A_b with
// A_b = a_q a_l for the pair b = (q <= l). Stored as CSR over rows a.
// hdiag[k] = Ho[k][k] (the diagonal one-body part, applied directly);
// hfull = Ho (M*M, row-major), used only for the one-particle space.
struct PairOp {
    const int *rowptr;      // P + 1
    const uint16_t *col;    // nnz
    const double2 *val;     // nnz
    const double2 *hdiag;   // M
    const double2 *hfull;   // M * M
    int nnz;
    // momentum-block form (nullptr unless Ht only couples pairs of equal q + l):
    // blocks K = 0 .. 2M-2 of the pairs (q, K-q), q = max(0,K-M+1) .. K/2, dense
    // row-major values in that order
    const double2 *hblk;
    int nhblk;
    int create_form;        // pair-creation kernel: 0 per-row tables in shared memory, 1 in registers
    int *status;            // device status word (1: a bounded wait timed out)
    // dense form (nullptr unless set): Ht as P x P row-major, for pair matrices with
    // no momentum-block or narrow block structure and P <= kGemmMaxP
    const double2 *hdense;
    // bounded waits of the warp-specialised dense product: limit in SM cycles
    // (0: the default, about two seconds) and a test switch that keeps its
    // gather warps from delivering any tile, so that the waits run out
    long long wait_cycles;
    int test_stall;
    // host copy of hblk (nhblk values) or null: the momentum kernel then takes
    // the block values as a kernel parameter (constant bank) instead of
    // staging them in shared memory
    const double2 *hblk_host;
    // fused launch plan of the space (order == nullptr: two kernels)
    FusedPlan fused;
    // direct form: momentum-block integrals applied row by row with no
    // intermediate (0 off, 1 on, 2 on for M <= kDirectAutoMaxM)
    int direct;
};

// The form a whole-vector H.psi (both stages, all rows) takes with op.
enum { kFormTwo = 0, kFormFused = 1, kFormDirect = 2 };
constexpr int kDirectAutoMaxM = 11;
int hpsi_form(const Space &sp, const PairOp &op);
constexpr int kGemmMaxP = 78;   // M <= 12: Ht (zero-padded to a multiple of 8 rows) fits shared memory

// Block-sparse form of the same pair matrix: when Ht decomposes into blocks
// (rows R_b x columns C_b, e.g. one block per total momentum for plane-wave
// orbitals) with every |C_b| <= kBlockCols, kernel 1 keeps each block's
// gathered column values in registers instead of staging all P of them.
// One packed buffer: int header [nblocks, ncols_total, nrows_total, nvals],
// then per block {col_begin, ncols, row_begin, nrows, val_begin}, then the
// columns (q | l << 8), then the rows (pair index a), then (8-byte aligned)
// the dense block values (row-major per block) as double2.
constexpr int kBlockCols = 16;
struct BlockOp {
    const int *prog;        // packed buffer (nullptr: not block-sparse)
    int bytes;              // size of the packed buffer
};

// Device tables of one space.
struct SpaceTables {
    const uint32_t *W;      // (M-1) x wstride, W[i*ws + p] = C(p+i, i+1) mod 2^32
    const double *sq;       // sqrt(n), n = 0 .. N+2
    // optional: occupations of every configuration of the space, occ_bits bits
    // per orbital (orbital k in bits [k*occ_bits, (k+1)*occ_bits)); kernels that
    // read it skip the index decode, null means decode
    const uint64_t *occ = nullptr;
    int occ_bits = 0;
    const uint64_t *occ2 = nullptr;   // the same for the (N-2)-particle space (occ_bits bits)
    const uint64_t *occ1 = nullptr;   // the same for the (N-1)-particle space (rho1; built on first use)
};
// Bits per orbital of the packed occupation table of an N-particle space (0:
// M orbitals do not fit in 64 bits).
int occ_bits_for(int N, int M);
cudaError_t launch_pack_occ(const Space &sp, const SpaceTables &tb, uint64_t *occ, int bits, cudaStream_t st);

// H.psi : out = H psi. E is scratch of P * nc2 complex (unused when N < 2).
// stages: bit 0 = kernel 1 (pair annihilation + pair matrix, writes E),
//         bit 1 = kernel 2 (pair creation, reads E, writes out); 3 = both.
// row0/row1: with the default shared-table creation kernel, only rows
// [row0, row1) of out are computed, into out[0 .. row1-row0) (psi stays the
// full vector); 0xffffffff = nc.
// m0/m1: with the momentum-block form, kernel 1 runs only over the
// (N-2)-configurations [m0, m1) -- the E columns a row range reads
// (launch_rows_mrange); other forms always run over the whole space.
cudaError_t launch_apply_h(const Space &sp, const SpaceTables &tb, const PairOp &op,
                           const BlockOp &bo, const double2 *psi, double2 *E, double2 *out,
                           cudaStream_t st, int stages = 3, uint32_t row0 = 0,
                           uint32_t row1 = 0xffffffffu, uint32_t m0 = 0, uint32_t m1 = 0xffffffffu);
// out[0], out[1] (device) = the lowest and highest (N-2)-configuration that
// rows [r0, r1) read in kernel 2.
cudaError_t launch_rows_mrange(const Space &sp, const SpaceTables &tb, uint32_t r0, uint32_t r1, uint32_t *out,
                               cudaStream_t st);

// Fused H.psi set-up: need[c] = the highest producer tile consumer tile c
// reads (device, ceil(nc / kFusedTile) entries); the persistent grid and
// dynamic shared memory of the fused kernel.
cudaError_t launch_fused_need(const Space &sp, const SpaceTables &tb, int *need, cudaStream_t st);
cudaError_t fused_config(const Space &sp, int *grid, size_t *smem);

// One member of a batched Lanczos, as the batched H.psi kernels see it
// (momentum-block pair matrix only).
struct BatchMember {
    Space sp;
    const uint32_t *W;
    const double *sq;
    const double2 *hblk;     // momentum-block pair matrix
    int nh;
    const double2 *hdiag;    // Ho[k][k]
    const double2 *lvec;     // Krylov basis, vector k at lvec + k * nc
    double2 *E;              // P x nc2 intermediate
    double2 *r;              // H.psi output (the Lanczos residual)
    const int *done;         // this member's breakdown flag
    const uint64_t *occ;     // packed occupations of the N and N-2 spaces (or null: decode)
    const uint64_t *occ2;
    int occ_bits;
};

// Batched H.psi for the members of one M: work1 / work2 list (member,
// block-in-member) for the annihilation / creation kernels; vec selects the
// Krylov vector each member applies H to. form: the two pair kernels
// (members need E), or the direct kernel over work2's row blocks with smem2
// = batch_smem(M, N, nh, 3) (real or complex block values).
enum { kBatchTwo = 0, kBatchDirectReal = 1, kBatchDirectComplex = 2 };
// Orbital counts up to which a batch takes the direct form (the single-space
// default's range).
constexpr int kBatchDirectMaxM = 11;
cudaError_t launch_batch_apply_h(int M, int form, const BatchMember *mem, const int2 *work1, int n1, size_t smem1,
                                 const int2 *work2, int n2, size_t smem2, int vec, cudaStream_t st);
// stage 1 / 2: the annihilation / creation kernels; 3: the direct kernel
size_t batch_smem(int M, int N, int nh, int stage);
// The direct form with real block values passed as a kernel parameter: up to
// batch_chunk_members(M) members per launch, their values in a host buffer of
// batch_vals_bytes(M) bytes filled slot by slot with batch_fill_vals (real
// parts of the member's momentum-block values); work lists (slot, block).
int batch_chunk_members(int M);
size_t batch_vals_bytes(int M);
void batch_fill_vals(int M, void *vals, int slot, int member, const double2 *hblk_host);
cudaError_t launch_batch_direct_vals(int M, const BatchMember *mem, const int2 *work, int n, size_t smem, int vec,
                                     const void *vals, cudaStream_t st);
// Sets the kernels' shared-memory limits (call outside stream capture).
cudaError_t batch_prepare(int M, size_t smem1, size_t smem2, size_t smem3);
// configurations per block of the batched kernels: stage 1 annihilation, 2 creation
int batch_rows_per_block(int stage);

// Densities as Gram matrices over the (N-order)-particle space:
// G[a][b] = sum_m conj(<m|A_a|phi>) <m|A_b|psi>, expanded to the reference
// layouts: order 1 -> rho1[k*M + l]; order 2 -> rho2[k + s*M + q*M^2 + l*M^3].
// partial: scratch of >= gram_partial_elems(sp, order) complex.
size_t gram_partial_elems(const Space &sp, int order);
// status / wait_cycles: the space's status word and the limit of the bounded
// waits of the tensor-core Gram kernel (0: about two seconds); test_stall
// keeps its gather warps from delivering any tile (testing the timeout path).
cudaError_t launch_density(const Space &sp, const SpaceTables &tb, int order,
                           const double2 *phi, const double2 *psi, double2 *partial,
                           double2 *out, cudaStream_t st, int *status = nullptr,
                           long long wait_cycles = 0, int test_stall = 0);

// Reference-layout tables built on the device.
cudaError_t launch_focks(const Space &sp, const SpaceTables &tb, int32_t *IF, cudaStream_t st);
cudaError_t launch_one_one_map(const Space &sp, const SpaceTables &tb, int32_t *Map,
                               cudaStream_t st);
// chunk counts per configuration (two_orbital = 0: v_k >= 2; 1: pairs k<s occupied)
cudaError_t launch_chunk_counts(const Space &sp, const SpaceTables &tb, int two_orbital,
                                int64_t *counts, cudaStream_t st);
// exclusive scan of counts * M*M into stride (int64), total chunks to *d_total
cudaError_t launch_stride_scan(const Space &sp, const int64_t *counts, int64_t *stride,
                               int64_t *d_total, void *scratch, size_t scratch_bytes,
                               size_t *scratch_needed, cudaStream_t st);
cudaError_t launch_two_map(const Space &sp, const SpaceTables &tb, int two_orbital,
                           const int64_t *stride, int32_t *Map, cudaStream_t st);
cudaError_t launch_narrow_stride(const int64_t *in, int32_t *out, int64_t n, cudaStream_t st);

// Lanczos vector kernels (all no-ops once *done != 0).
struct LanczosState {
    double2 *alpha;      // lm
    double *beta;        // lm
    double *maxbeta;     // 1
    int *done;           // 1
    int *iters;          // 1 : steps completed (lm unless broken down)
    double2 *coef;       // lm   : reorthogonalisation coefficients of the current step
    double2 *partial;    // scratch of lanczos_partial_elems(nc, lm) complex
    int nparts;          // = lanczos_parts(nc): blocks of the fixed-size reductions
};

int lanczos_parts(int64_t nc);
size_t lanczos_partial_elems(int64_t nc, int lm);
cudaError_t launch_lanczos_start(const double2 *v0, const double2 *hv, double2 *r, int64_t nc,
                                 LanczosState s, cudaStream_t st);
cudaError_t launch_lanczos_beta(int i, int lm, double tol, LanczosState s, cudaStream_t st);
cudaError_t launch_lanczos_scale(const double2 *r, double2 *vnext, int64_t nc, int i,
                                 LanczosState s, cudaStream_t st);
cudaError_t launch_lanczos_alpha(const double2 *vprev, const double2 *vcur, double2 *r,
                                 int64_t nc, int i, LanczosState s, cudaStream_t st);
cudaError_t launch_lanczos_reorth(const double2 *V, int nvec, double2 *r, int64_t nc, int i,
                                  LanczosState s, cudaStream_t st);
cudaError_t launch_combine(const double2 *V, int nvec, int64_t nc, const double *z,
                           double2 *out, cudaStream_t st);
cudaError_t launch_lanczos_no_reorth(const double2 *vcur, double2 *r, int64_t nc, int i, LanczosState s,
                                     cudaStream_t st);
cudaError_t launch_axpy_real(double2 *acc, const double2 *v, int64_t nc, const double *z, int first,
                             cudaStream_t st);
cudaError_t launch_lanczos_axpy(const double2 *vprev, double2 *r, int64_t nc, int i, LanczosState s,
                               cudaStream_t st);
cudaError_t launch_dot(const double2 *a, const double2 *b, int64_t nc, double2 *partial,
                       double2 *result, cudaStream_t st);

// Row-shard primitives of a sharded Lanczos (n rows of this rank; scalars on the
// device; every kernel returns at entry once *done != 0). The caller sums the
// per-rank results (dot, coef, norm2) over the ranks between the calls.
size_t shard_scratch_elems(int64_t n, int lm);
cudaError_t launch_shard_scale(int64_t n, const double2 *r, double2 *vnext, const double *beta_i, const int *done,
                               cudaStream_t st);
cudaError_t launch_shard_axpy_dot(int64_t n, const double2 *vprev, const double2 *vcur, double2 *r,
                                  const double *beta_i, double2 *scratch, double2 *dot, const int *done,
                                  cudaStream_t st);
cudaError_t launch_shard_multidot(int64_t n, const double2 *V, int nvec, const double2 *r, const double2 *vcur,
                                  const double2 *alpha, double2 *scratch, double2 *coef, const int *done,
                                  cudaStream_t st);
cudaError_t launch_shard_update(int64_t n, const double2 *V, int nvec, double2 *r, const double2 *vcur,
                                const double2 *alpha, const double2 *coef, double2 *scratch, double *norm2,
                                const int *done, cudaStream_t st);
cudaError_t launch_shard_beta(int i, double tol, const double *norm2, double *beta, double *maxbeta, int *done,
                              int *iters, cudaStream_t st);

}  // namespace mcpi
