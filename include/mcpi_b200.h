/* mcpi_b200 -- native C ABI of the B200 multiconfigurational hot path.
 *
 * One "space" is the Fock space of N bosons in M orbitals (1 <= M <= 16,
 * NC(N,M) = C(N+M-1,N) < 2^31) resident on one CUDA device. Every array
 * argument named d_* is a device pointer; complex numbers are two doubles
 * (re, im), layout-compatible with C99 `double complex`, std::complex<double>
 * and cuDoubleComplex. Work is enqueued on the space's stream and is complete
 * after mcpi_space_sync() (functions returning host results synchronise).
 * Every function returns MCPI_OK or an error code; mcpi_last_error() gives a
 * message for the calling thread. Nothing aborts the process.
 *
 * Reference counterparts (andriati-alex/mcpi, file:line) are named beside each
 * entry point. The reference-named drop-in interface (NC, setupFocks,
 * applyHconf_XX, OBrho_XM, TBrho_XX, ...) is declared in mcpi_dropin.h and
 * implemented on top of this one.
 */
#ifndef MCPI_B200_H
#define MCPI_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MCPI_API __attribute__((visibility("default")))
#else
#define MCPI_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MCPI_OK 0
#define MCPI_ERR_ARG 1          /* invalid argument (sizes, NULL pointers) */
#define MCPI_ERR_RANGE 2        /* NC(N,M) or a table size exceeds the supported range */
#define MCPI_ERR_CUDA 3         /* a CUDA runtime call failed */
#define MCPI_ERR_NOMEM 4        /* device or host allocation failed */
#define MCPI_ERR_STATE 5        /* call order (e.g. no integrals set) */
#define MCPI_ERR_NUMERIC 6      /* tridiagonal eigensolver did not converge */
#define MCPI_ERR_TIMEOUT 7      /* a kernel's bounded wait expired (its output is invalid) */

/* variants of the two-body folding (see mcpi_set_integrals) */
#define MCPI_VARIANT_MAPS 0     /* applyHconf_X / _XX / _omp and the CUDA kernel */
#define MCPI_VARIANT_HASH 1     /* applyHconf (plain): Rule 9 summed over all orderings */

typedef struct mcpi_space_s *mcpi_space;

MCPI_API const char *mcpi_status_string(int status);
MCPI_API const char *mcpi_last_error(void);

/* NC(N,M) = C(N+M-1, N), exact (configurationsMap.h:145-202, NC). */
MCPI_API int mcpi_nc(int N, int M, int64_t *nc);

/* Create / destroy a space on `device` (configurationsMap.h:206-344 state:
 * NCmat + IF tables; here only the binomial table W and sqrt table are kept). */
MCPI_API int mcpi_space_create(int N, int M, int device, mcpi_space *out);
MCPI_API int mcpi_space_destroy(mcpi_space sp);
/* Enqueue all further work of the space on `stream` (a cudaStream_t; NULL is the
 * legacy default stream). A new space uses a private non-blocking stream. */
MCPI_API int mcpi_space_set_stream(mcpi_space sp, void *stream);
MCPI_API int mcpi_space_sync(mcpi_space sp);
/* Space options. MCPI_OPT_DENSE_PAIR_KERNEL (value 0/1): always use a dense
 * pair-matrix kernel for H.psi even when the integrals decompose into small
 * blocks (takes effect at the next mcpi_set_integrals). */
#define MCPI_OPT_DENSE_PAIR_KERNEL 1
/* MCPI_OPT_NO_MOMENTUM_KERNEL (0/1): do not use the momentum-block kernel
 * (chosen when the pair matrix only couples pairs of equal total orbital index,
 * as plane-wave integrals of a translation-invariant interaction do). */
#define MCPI_OPT_NO_MOMENTUM_KERNEL 2
/* MCPI_OPT_CREATE_FORM: form of the pair-creation kernel of H.psi -- 0 per-row
 * tables in shared memory (default), 1 per-row tables in registers. Takes
 * effect at the next mcpi_set_integrals. */
#define MCPI_OPT_CREATE_FORM 3
/* MCPI_OPT_NO_GEMM_KERNEL (0/1): general (dense) pair matrices use the
 * compressed-row kernel instead of the register-tiled dense product (which is
 * otherwise chosen for M <= 12). Takes effect at the next mcpi_set_integrals. */
#define MCPI_OPT_NO_GEMM_KERNEL 4
/* MCPI_OPT_WAIT_LIMIT_KCYCLES (>= 0): limit, in thousands of SM cycles, of
 * each bounded wait inside the warp-specialised dense-product kernel (0, the
 * default: about two seconds). A wait that runs out makes the kernel return
 * and the next synchronising call report MCPI_ERR_TIMEOUT. */
#define MCPI_OPT_WAIT_LIMIT_KCYCLES 5
/* MCPI_OPT_TEST_STALL_GATHER (0/1): for testing the timeout paths only — the
 * gather warps of the dense-product and tensor-core Gram kernels deliver no
 * tile and the fused H.psi kernel's producers never count themselves done, so
 * the waits run out (results are invalid while it is set). */
#define MCPI_OPT_TEST_STALL_GATHER 6
/* MCPI_OPT_NO_OCC_TABLES (0/1): build no packed occupation tables (the H.psi
 * kernels then decode every row index; 1 also frees existing tables). Takes
 * effect at the next mcpi_set_integrals. */
#define MCPI_OPT_NO_OCC_TABLES 7
/* MCPI_OPT_FUSED_HPSI (0/1, default 0): run H.psi with momentum-block
 * integrals as one persistent kernel that interleaves the pair-annihilation
 * and pair-creation tiles, so most of the P x NC(N-2,M) intermediate is read
 * back from L2 instead of HBM (results are bitwise those of the two-kernel
 * form; at N=16, M=10 it is slower: 0.365 against 0.300 ms). Whole-vector
 * calls only; row ranges keep the two kernels. */
#define MCPI_OPT_FUSED_HPSI 8
/* MCPI_OPT_FUSED_LEAD (>= 0, default 128): producer tiles (256
 * configurations of the N-2 space each) the fused kernel's schedule runs
 * ahead of its consumers. */
#define MCPI_OPT_FUSED_LEAD 9
/* MCPI_OPT_DIRECT_HPSI: apply momentum-block integrals row by row, gathering
 * every term straight from the state, with no P x NC(N-2,M) intermediate
 * (N < 64; whole vectors and row ranges alike).
 * 0 off, 1 on, 2 (default) on for M <= 11, where it is the faster form. */
#define MCPI_OPT_DIRECT_HPSI 11
MCPI_API int mcpi_space_set_option(mcpi_space sp, int option, int value);
MCPI_API int mcpi_space_dims(mcpi_space sp, int *N, int *M, int64_t *nc);
/* Device memory on the space's device, and a synchronous copy in any direction
 * (host or device pointers, on the space's stream), for hosts without CUDA
 * headers. Replace the reference's malloc'd arrays that must live on the GPU
 * (configurationsMap.h:46-116 rarrDef/carrDef/iarrDef). */
MCPI_API int mcpi_alloc(mcpi_space sp, size_t bytes, void **d_ptr);
MCPI_API int mcpi_free(mcpi_space sp, void *d_ptr);
MCPI_API int mcpi_memcpy(mcpi_space sp, void *dst, const void *src, size_t bytes);

/* ---- tables in the reference layouts, built on the device ---------------- */
/* NCmat[n + (N+1)*m] = NC(n,m), host output (configurationsMap.h:206-234). */
MCPI_API int mcpi_ncmat(int N, int M, int32_t *h_ncmat);
/* index <-> occupations, host scalars (configurationsMap.h:238-305). */
MCPI_API int mcpi_index_to_fock(int N, int M, int64_t index, int32_t *h_v);
MCPI_API int mcpi_fock_to_index(int N, int M, const int32_t *h_v, int64_t *index);
/* IF[j + i*M] (configurationsMap.h:309-344, setupFocks), nc*M int32. */
MCPI_API int mcpi_focks(mcpi_space sp, int32_t *d_IF);
/* Map[i + k*nc + l*M*nc] (configurationsMap.h:348-417, OneOneMap), nc*M*M int32. */
MCPI_API int mcpi_one_one_map(mcpi_space sp, int32_t *d_map);
/* Number of int32 entries of MapOT (two_orbital=0, configurationsMap.h:617-664)
 * or MapTT (two_orbital=1, configurationsMap.h:421-474). */
MCPI_API int mcpi_two_map_size(mcpi_space sp, int two_orbital, int64_t *entries);
/* MapOT / MapTT and their strides (configurationsMap.h:668-762 / 478-613);
 * d_stride: nc int64 entries (the reference's strideC, widened). */
MCPI_API int mcpi_two_map(mcpi_space sp, int two_orbital, int64_t *d_stride, int32_t *d_map);

/* ---- operators -------------------------------------------------------------- */
/* Orbital integrals, host arrays: Ho[k*M + l] = Ho(k,l) (M*M complex),
 * Hint[k + s*M + q*M^2 + l*M^3] (M^4 complex) = coefficient of a+_k a+_s a_q a_l.
 * variant selects the reference's folding of the two-body sum
 * (hamiltonianMatrix.h:391-416 vs :1370-1418); both agree when Hint has the
 * bosonic 8-fold symmetry. Builds the forward and adjoint pair operators. */
MCPI_API int mcpi_set_integrals(mcpi_space sp, const double *h_Ho, const double *h_Hint, int variant);
/* out = H C (hamiltonianMatrix.h:891-1425 applyHconf_XX semantics; _omp, _X and
 * the CUDA applyHconf kernel compute the same; MCPI_VARIANT_HASH gives applyHconf). */
MCPI_API int mcpi_apply_h(mcpi_space sp, const void *d_C, void *d_out);
/* out_k = H C_k for k = 0 .. count-1 with C_k and out_k in HOST memory (nc
 * complex doubles each; page-locked memory from cudaHostAlloc or
 * cudaHostRegister gets full PCIe bandwidth). The states stream through two
 * device buffer pairs held by the space: the copy in of state k+1, H.psi of
 * state k and the copy out of state k-1 run concurrently on three streams.
 * Returns when every out_k is written. The same result as count calls of the
 * reference's applyHconf* on host arrays (hamiltonianMatrix.h:891-1425), which
 * copy and compute one state at a time. */
MCPI_API int mcpi_apply_h_host(mcpi_space sp, int count, const void *const *h_C, void *const *h_out);
/* Rows [row0, row1) of H C into d_out[0 .. row1-row0), d_C being the whole
 * vector: the local part of a row-sharded H.psi (each rank owns a row block
 * and gathers the full vector first). Needs N >= 2. No reference counterpart.
 * With momentum-block integrals the pair-annihilation kernel runs only over
 * the (N-2)-configurations these rows read (found on the first call for a row
 * block, which synchronises the space's stream once). */
MCPI_API int mcpi_apply_h_rows(mcpi_space sp, const void *d_C, int64_t row0, int64_t row1, void *d_out);
/* mcpi_apply_h, timed: runs it reps times with CUDA events around each of its
 * two kernels on the space's stream (synchronising after every repetition) and
 * returns their mean durations in ms: h_ms[0] pair annihilation + pair-matrix
 * kernel, h_ms[1] pair creation kernel (where the call takes the direct or
 * the fused one-kernel form: h_ms[0] that kernel, h_ms[1] = 0). For
 * measurement, not for production. */
MCPI_API int mcpi_apply_h_profile(mcpi_space sp, const void *d_C, void *d_out, int reps, float *h_ms);
/* out = H C without allocating anything. No counterpart in the reference.
 * For callers that cannot allocate device memory where they need H.psi (a
 * host whose own pool allocator owns the GPU's memory, or a loop that cannot
 * absorb cudaMalloc's synchronisation): it runs the H.psi kernels with all
 * scratch taken from a 32 MiB array compiled into the library, which every GPU
 * that loads the library holds until the process exits. Host integrals as in
 * mcpi_set_integrals, device vectors d_C / d_out (nc complex), work enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream). Returns
 * MCPI_ERR_RANGE, with nothing enqueued, when M > 10, N > 64 or the tables plus
 * the P * NC(N-2,M) intermediate exceed the array (at M = 10: N <= 10).
 * Calls share the array: calls that overlap on the GPU race. The first call
 * on a device looks up the array's device address; make it before any stream
 * capture begins. Not capturable: a call on a capturing stream (or on the
 * legacy stream while another stream captures) returns MCPI_ERR_ARG with
 * nothing enqueued. Each call folds the integrals on the calling thread's
 * stack, about 58 KB at M = 10. */
MCPI_API int mcpi_apply_h_static(int N, int M, const double *h_Ho, const double *h_Hint, int variant,
                                 const void *d_C, void *d_out, void *stream);
/* out = H^dagger C (adjoint of the operator above; equal to H C when Ho is
 * Hermitian and Hint has the 8-fold symmetry). No reference counterpart. */
MCPI_API int mcpi_apply_h_adjoint(mcpi_space sp, const void *d_C, void *d_out);
/* rho1[k*M + l] = <a+_k a_l> (onebodyMatrix.h:190-251, OBrho_XM), device output M*M. */
MCPI_API int mcpi_rho1(mcpi_space sp, const void *d_C, void *d_rho1);
/* rho2[k + s*M + q*M^2 + l*M^3] = <a+_k a+_s a_q a_l> (twobodyMatrix.h:991-1487, TBrho_XX). */
MCPI_API int mcpi_rho2(mcpi_space sp, const void *d_C, void *d_rho2);
/* Transition densities <phi|a+_k a_l|psi> (t1[k*M + l]) and
 * <phi|a+_k a+_s a_q a_l|psi> (t2, rho2 layout): every entry reduced, valid for
 * phi != psi. Generalise OBrho_XM / TBrho_XX; no reference counterpart. */
MCPI_API int mcpi_trans_rho1(mcpi_space sp, const void *d_phi, const void *d_psi, void *d_t1);
MCPI_API int mcpi_trans_rho2(mcpi_space sp, const void *d_phi, const void *d_psi, void *d_t2);
/* <a, b> = sum conj(a) b (groundStateLieb.c:73-85, carrDot), host result. */
MCPI_API int mcpi_dot(mcpi_space sp, const void *d_a, const void *d_b, double *h_result2);

/* Row-shard Lanczos primitives. No counterpart in the reference, whose
 * lanczos (groundStateLieb.c:217-344) runs in one process: here a process per
 * GPU owns rows [row0, row1) of every Krylov vector (n = row1 - row0, its
 * shard) and runs the reference's recurrence with these calls, summing each
 * per-rank result (dot, coefficients, norm^2) over the ranks with an
 * all-reduce between the calls (mcpi_b200/distributed.py is the driver; the
 * H.psi of a shard is mcpi_apply_h_rows on the all-gathered vector). All
 * scalars stay in device memory, so a solve needs no host round trip; every
 * kernel returns at entry once *d_done != 0, so all ranks keep issuing the
 * same collectives after a breakdown. Sums inside a rank run in a fixed
 * order. Device pointers (complex = 2 doubles), work on `stream`.
 *   scratch: mcpi_shard_scratch_elems(n, lm) complex entries. */
MCPI_API size_t mcpi_shard_scratch_elems(int64_t n, int lm);
/* vnext = r / *beta_i */
MCPI_API int mcpi_shard_scale(int64_t n, const void *d_r, void *d_vnext, const double *d_beta_i,
                              const int *d_done, void *stream);
/* r -= *beta_i vprev (skipped when d_vprev is NULL); *d_dot = <vcur, r> over the shard */
MCPI_API int mcpi_shard_axpy_dot(int64_t n, const void *d_vprev, const void *d_vcur, void *d_r,
                                 const double *d_beta_i, void *d_scratch, void *d_dot, const int *d_done,
                                 void *stream);
/* coef[j] = <V_j, r - alpha vcur> over the shard, j < nvec (V: nvec shards of n) */
MCPI_API int mcpi_shard_multidot(int64_t n, const void *d_V, int nvec, const void *d_r, const void *d_vcur,
                                 const void *d_alpha, void *d_scratch, void *d_coef, const int *d_done,
                                 void *stream);
/* r = r - alpha vcur - sum_j coef[j] V_j (nvec may be 0); *d_norm2 = |r|^2 over the shard */
MCPI_API int mcpi_shard_update(int64_t n, const void *d_V, int nvec, void *d_r, const void *d_vcur,
                               const void *d_alpha, const void *d_coef, void *d_scratch, double *d_norm2,
                               const int *d_done, void *stream);
/* beta[i] = sqrt(*d_norm2) (summed over the ranks) and the breakdown test of
 * groundStateLieb.c:287-292: sets *d_done = 1 and *d_iters = i */
MCPI_API int mcpi_shard_beta(int i, double tol, const double *d_norm2, double *d_beta, double *d_maxbeta,
                             int *d_done, int *d_iters, void *stream);
/* out = sum_k V_k z[k], k < nvec (z real, device) -- a shard of the Ritz vector */
MCPI_API int mcpi_shard_combine(int64_t n, const void *d_V, int nvec, const double *d_z, void *d_out,
                                void *stream);

/* ---- Lanczos (groundStateLieb.c:217-471) ------------------------------------ */
/* Lanczos with full classical Gram-Schmidt reorthogonalisation
 * (groundStateLieb.c:217-344, lanczos). d_lvec holds lm vectors of nc complex,
 * d_lvec[0..nc) = start vector on entry. h_diag (lm complex, alpha) and
 * h_offdiag (lm doubles, beta) receive the tridiagonal; *iters the number of
 * steps done (lm, or the step of a breakdown beta_i/max beta < 1e-15). */
MCPI_API int mcpi_lanczos(mcpi_space sp, void *d_lvec, int lm, double *h_diag, double *h_offdiag,
                 int *iters);
/* Lowest eigenpair of H from niter Lanczos steps started at d_C
 * (groundStateLieb.c:348-471, ground). d_C receives the Ritz vector; *E0 the
 * eigenvalue. The niter*nc Krylov basis (and mcpi_lanczos's small state and
 * residual) are workspaces of the space: allocated at the first call that needs
 * them, reused by later calls, grown when a call needs more, freed by
 * mcpi_space_destroy. */
MCPI_API int mcpi_ground(mcpi_space sp, void *d_C, int niter, double *E0, int *iters);
/* mcpi_ground for spaces whose niter x nc Krylov basis does not fit: plain
 * three-term Lanczos (no reorthogonalisation; same breakdown rule) in two
 * passes, the second regenerating the Krylov vectors -- bitwise the same, all
 * reductions being deterministic -- to accumulate the Ritz vector. Holds four
 * vectors of nc. Without reorthogonalisation the Lanczos matrix can acquire
 * spurious copies of converged eigenvalues; the lowest one is unaffected. */
MCPI_API int mcpi_ground_lowmem(mcpi_space sp, void *d_C, int niter, double *E0, int *iters);
/* Eigenvalues (ascending, into d) and optionally row-major eigenvectors
 * z[k*n + j] of the symmetric tridiagonal (d, e): the LAPACKE_dstev('V') contract
 * used at groundStateLieb.c:435. Host arrays. */
MCPI_API int mcpi_tridiag_eig(int n, double *d, double *e, double *z);

/* ---- batched ground states (no reference counterpart) ----------------------- */
/* Many Lanczos ground-state solves of different (N, M) in one device arena,
 * advanced together and replayed as one CUDA graph: each Lanczos stage is one
 * launch over all members, every member keeps the reference recurrence
 * (groundStateLieb.c:217-344: full CGS reorthogonalisation, breakdown test),
 * and the lowest eigenvalue of each tridiagonal is found on the device by
 * Sturm bisection. lm = Lanczos steps per member (2 .. 2048). Members need
 * N >= 2, 2 <= M <= 16 and integrals that conserve the total orbital index
 * (plane-wave integrals of a translation-invariant interaction, e.g.
 * mcpi_lieb_integrals). The batch changes the calling thread's current device. */
typedef struct mcpi_batch_s *mcpi_batch;
MCPI_API int mcpi_batch_create(int count, const int *N, const int *M, int lm, int device, mcpi_batch *out);
MCPI_API int mcpi_batch_member_size(mcpi_batch b, int member, int64_t *nc);
MCPI_API int mcpi_batch_set_integrals(mcpi_batch b, int member, const double *h_Ho, const double *h_Hint,
                                      int variant);
/* Start vector of a member (host or device pointer, nc complex); kept for
 * every later mcpi_batch_run. */
MCPI_API int mcpi_batch_set_start(mcpi_batch b, int member, const void *C);
/* Runs all members (the first call captures and instantiates the graph) and
 * returns each member's lowest eigenvalue and Lanczos step count. */
MCPI_API int mcpi_batch_run(mcpi_batch b, double *h_E0, int *h_iters);
MCPI_API int mcpi_batch_arena_bytes(mcpi_batch b, size_t *bytes);
/* Tile schedule of the batch's vector stages (rows of one member per work tile:
 * 512, 1024 or 2048). 0 (the default) lets the first mcpi_batch_run time one
 * Lanczos step's vector stages with each tile on this batch's own arena and
 * keep the fastest (the autotuner); a fixed value pins it, e.g. to reproduce
 * results bit for bit across processes (the tile sets the reduction order).
 * Only before the first mcpi_batch_run. No reference counterpart. */
MCPI_API int mcpi_batch_set_schedule(mcpi_batch b, int tile_rows);
/* The tile in use (0 before the first run) and, when it was autotuned, the
 * probe time of each candidate 512 / 1024 / 2048 in h_ms[0..2] (ms; may be NULL). */
MCPI_API int mcpi_batch_schedule(mcpi_batch b, int *tile_rows, float *h_ms);
/* Schedule of the batched H.psi: bit 0 runs the groups of members with the
 * same M as concurrent graph branches (else one after another), bit 1 hands
 * out their blocks interleaved across members (else member by member). -1
 * (the default) lets the first mcpi_batch_run time one batched H.psi under
 * each of the four schedules on this batch's own arena and keep the fastest;
 * no schedule changes any member's arithmetic. Only before the first run. No
 * reference counterpart. */
MCPI_API int mcpi_batch_set_hpsi_schedule(mcpi_batch b, int schedule);
/* The H.psi schedule in use (-1 before the first run) and the probe time of
 * each schedule 0..3 in h_ms[0..3] when it was autotuned (ms; may be NULL). */
MCPI_API int mcpi_batch_hpsi_schedule(mcpi_batch b, int *schedule, float *h_ms);
MCPI_API int mcpi_batch_destroy(mcpi_batch b);

/* ---- model inputs ------------------------------------------------------------ */
/* Lieb-Liniger plane-wave integrals on a ring of length L
 * (groundStateLieb.c:129-213, setupHo / setupHint), host outputs. */
MCPI_API int mcpi_lieb_integrals(int M, double g, double L, double *h_Ho, double *h_Hint);

#ifdef __cplusplus
}
#endif

#endif /* MCPI_B200_H */
