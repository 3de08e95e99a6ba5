// H.psi on the device.
//
// Reference semantics: hamiltonianMatrix.h (applyHconf / _X / _XX / _omp) and
// cuda/hamiltonianMatrix.cuh:60-626 compute, row by row,
//     out = sum_kl Ho[k][l] a+_k a_l psi + 1/2 sum Hint[k,s,q,l] a+_k a+_s a_q a_l psi
// through nine rule families that each read one representative Hint entry
// (the pair matrix built on the host, capi.cpp build_pair_op, reproduces that
// folding exactly, for any Hint).
//
// B200 formulation. Every two-body term factors through the (N-2)-particle
// space: with pairs a = (k<=s), b = (q<=l) and A_b = a_q a_l,
//     H2 psi = sum_a A+_a  E_a,     E_a(m) = sum_b Ht[a][b] <m|A_b|psi>.
// Kernel 1 (one thread per (N-2)-configuration m) gathers the P = M(M+1)/2
// values <m|A_b|psi> = c_b(m) psi[index(m + e_q + e_l)] straight into shared
// memory with cp.async, applies the sparse pair matrix, and writes E[a][m]
// (pair-major, so consecutive m give coalesced stores). Kernel 2 (one thread
// per N-configuration i) gathers E[a][index(v_i - e_k - e_s)] for its occupied
// pairs, adds the diagonal one-body term, and writes out[i]. Off-diagonal
// one-body terms are folded into Ht on the host (a+_k a_l = (N-1)^-1 sum_s
// a+_k a+_s a_s a_l on N particles). Every E entry is written once and read
// once, so the HBM traffic per H.psi is psi + out + 2 * P * nc2 * 16 bytes,
// against the reference's nc*M^2 + map chunks of int32 indices; the psi
// gathers of kernel 1 are served from L2 (psi is 32.7 MB at N=16, M=10).
// All jump indices come from the prefix-table hash in fock.cuh (no maps).
#include <cuda_runtime.h>
#include "fock.cuh"
#include "kernels.h"
#include "mbarrier.cuh"

namespace mcpi {

namespace {

constexpr int kT1 = 64;    // threads (= (N-2)-configurations) per block, kernel 1 (compressed-row form)
constexpr int kCsrStaged = 1024;   // pair-matrix nonzeros staged in shared memory
constexpr int kT2 = 256;   // threads per block, kernel 2 (register form) and kernel 1 (momentum form)
constexpr int kTC = 256;   // threads (= rows) per block, kernel 2 (shared-table form)
constexpr int kCreateBatch = 8;   // E gathers issued together per thread, kernel 2 (shared-table form)

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// the same, cached in L2 only (scattered 16-byte gathers with no L1 reuse)
__device__ __forceinline__ void cp_async16_cg(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n"
                 "cp.async.wait_group 0;\n" ::
                     : "memory");
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

// Loads the W table and sqrt table of the space into shared memory.
__device__ __forceinline__ void load_tables(const Space &sp, const SpaceTables &tb, uint32_t *W,
                                            double *sq)
{
    int nw = (sp.M - 1) * sp.wstride;
    for (int x = threadIdx.x; x < nw; x += blockDim.x) W[x] = tb.W[x];
    for (int x = threadIdx.x; x < sp.wstride; x += blockDim.x) sq[x] = tb.sq[x];
}

// ---------------------------------------------------------------------------
// kernel 1: E[a][m] = sum_b Ht[a][b] c_b(m) psi[index(m + pair b)]
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kT1) k_pair_annihilate(Space sp, SpaceTables tb, PairOp op,
                                                         const double2 *__restrict__ psi,
                                                         double2 *__restrict__ E)
{
    constexpr int P = M * (M + 1) / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *D = reinterpret_cast<double2 *>(smem_raw);             // P x kT1
    double2 *hv = D + P * kT1;                                      // nnz (when staged)
    double *sq = reinterpret_cast<double *>(hv + (op.nnz <= kCsrStaged ? op.nnz : 0));
    int *rp = reinterpret_cast<int *>(sq + sp.wstride);             // P + 1
    int *cl = rp + P + 1;                                           // nnz (when staged)
    uint32_t *W = reinterpret_cast<uint32_t *>(cl + (op.nnz <= kCsrStaged ? op.nnz : 0));
    load_tables(sp, tb, W, sq);
    const bool staged = op.nnz <= kCsrStaged;
    for (int x = threadIdx.x; x <= P; x += blockDim.x) rp[x] = op.rowptr[x];
    if (staged)
        for (int x = threadIdx.x; x < op.nnz; x += blockDim.x) {
            hv[x] = op.val[x];
            cl[x] = op.col[x];
        }
    __syncthreads();

    const int t = threadIdx.x;
    const uint32_t m = blockIdx.x * kT1 + t;
    if (m >= sp.nc2) return;
    const int ws = sp.wstride;

    int u[M], Q[M];
    occupations<M>(tb.occ2, tb.occ_bits, m, sp.N - 2, sp.nc2, W, ws, u, Q);
    uint32_t B0[M], B1[M], B2[M];
    prefix_table<M>(Q, 0, W, ws, B0);
    prefix_table<M>(Q, 1, W, ws, B1);
    prefix_table<M>(Q, 2, W, ws, B2);

    double2 *Dt = D + t;
#pragma unroll
    for (int q = 0; q < M; ++q)
#pragma unroll
        for (int l = q; l < M; ++l) {
            const uint32_t j = idx_add2(sp.nc, B0, B1, B2, q, l, M);
            cp_async16(Dt + pair_index(q, l, M) * kT1, psi + j);
        }
    cp_async_wait_all();
    // <m|a_q a_l|psi> = sqrt((u_q+1)(u_l+1)) psi_j  (q<l),  sqrt((u_q+1)(u_q+2)) psi_j  (q=l)
#pragma unroll
    for (int q = 0; q < M; ++q)
#pragma unroll
        for (int l = q; l < M; ++l) {
            const double c = (q == l) ? sq[u[q] + 1] * sq[u[q] + 2] : sq[u[q] + 1] * sq[u[l] + 1];
            double2 &d = Dt[pair_index(q, l, M) * kT1];
            d.x *= c;
            d.y *= c;
        }
    const size_t stride = sp.nc2;
    for (int a = 0; a < P; ++a) {
        const int z0 = rp[a], z1 = rp[a + 1];
        double2 e = make_double2(0.0, 0.0);
        if (staged) {
            for (int z = z0; z < z1; ++z) cfma(e, hv[z], Dt[cl[z] * kT1]);
        } else {
            for (int z = z0; z < z1; ++z) cfma(e, __ldg(op.val + z), Dt[__ldg(op.col + z) * kT1]);
        }
        E[a * stride + m] = e;
    }
}

// ---------------------------------------------------------------------------
// kernel 1, dense-product form for general pair matrices (P <= kGemmMaxP), on
// the FP64 tensor cores (mma.sync m16n8k4 .f64: 16 x 8 x 4 per warp instruction).
// A persistent block keeps Ht in shared memory. Per tile of kGM
// (N-2)-configurations it gathers D[b][m] = c_b(m) psi[index(m + pair b)] into
// shared memory (cp.async), then forms E^T[m][a] = sum_b D^T[m][b] Ht^T[b][a]:
// MMA rows are configurations, columns pairs a, the reduction runs over pairs b.
// A warp owns 16 configurations and a range of 8-pair column tiles; per step of
// 4 b it loads two complex D entries and one complex Ht entry per column tile
// per lane (16-byte loads, conflict-free by XOR swizzles of the column index)
// and forms the complex product from three real ones,
//   t1 += Dr Hr,  t2 += Di Hi,  t3 += (Dr + Di)(Hr + Hi);  Er = t1 - t2, Ei = t3 - t1 - t2,
// which saves a quarter of the MMAs. The accumulator layout puts 8 consecutive
// configurations of one a in a lane quad's rows, so each E store instruction
// writes four full 128-byte rows.
// Per configuration: P gathers, 3 P^2 FP64 multiply-adds on the tensor cores
// (4 P^2 algorithmic), P stores.
// Shared layout (complex entries unless noted):
//   Hs[a][b ^ ((a & 1) << 2)]   PA x HS, zero outside a < P, b < P
//   D[b][m ^ ((b & 3) << 1)]    PK x kGM, rows b >= P zero
//   Cs[b][m ^ ((b & 3) << 2)]   PK x kGM doubles (warp-specialised form with
//                               the scaling in the product warps), rows b >= P zero
// ---------------------------------------------------------------------------
constexpr int kTG = 256;   // threads per block, dense-product form
constexpr int kGM = 64;    // (N-2)-configurations per tile (4 MMA row groups of 16)

// m16n8k4: A 16 x 4 (a0 row g, a1 row g + 8; column t), B 4 x 8 (row t, column g),
// C 16 x 8 (c0, c1 row g, c2, c3 row g + 8; columns 2t, 2t + 1), g = lane / 4, t = lane % 4
__device__ __forceinline__ void dmma16(double (&c)[4], double a0, double a1, double b)
{
    asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, {%0, %1, %2, %3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b));
}

template <int M>
struct GemmShape {
    static constexpr int P = M * (M + 1) / 2;
    static constexpr int PA = (P + 7) / 8 * 8;     // a padded to whole 8-column MMA tiles
    static constexpr int PK = (P + 3) / 4 * 4;     // b padded to whole 4-deep MMA steps
    static constexpr int HS = (PK + 7) / 8 * 8;    // row stride of Hs (a multiple of 8 for the swizzle)
    static constexpr int NT = PA / 8;
    static constexpr size_t hbytes = sizeof(double2) * (size_t)PA * HS;
    static constexpr size_t dbytes = sizeof(double2) * (size_t)PK * kGM;
};

// Gather of one tile's D (this thread's share: configuration cfg, pairs b with
// b % kParts == part) as cp.async copies into D, committed as one group; the
// occupations u of the configuration are returned for the scaling once the
// copies have landed. Configurations past nc2 get zero rows.
template <int M, int kParts>
__device__ __forceinline__ void gemm_gather(const Space &sp, const SpaceTables &tb, const uint32_t *W,
                                            const double2 *__restrict__ psi, double2 *D, uint32_t m, int cfg,
                                            int part, int (&u)[M])
{
    constexpr int P = M * (M + 1) / 2;
    if (m < sp.nc2) {
        int Q[M];
        occupations<M>(tb.occ2, tb.occ_bits, m, sp.N - 2, sp.nc2, W, sp.wstride, u, Q);
        uint32_t B0[M], B1[M], B2[M];
        prefix_table<M>(Q, 0, W, sp.wstride, B0);
        prefix_table<M>(Q, 1, W, sp.wstride, B1);
        prefix_table<M>(Q, 2, W, sp.wstride, B2);
#pragma unroll
        for (int q = 0; q < M; ++q)
#pragma unroll
            for (int l = q; l < M; ++l) {
                const int pb = pair_index(q, l, M);
                if (pb % kParts == part) {
                    const uint32_t j = idx_add2(sp.nc, B0, B1, B2, q, l, M);
                    cp_async16_cg(D + pb * kGM + (cfg ^ ((pb & 3) << 1)), psi + j);
                }
            }
    } else {
#pragma unroll
        for (int i = 0; i < M; ++i) u[i] = 0;
        for (int pb = part; pb < P; pb += kParts) D[pb * kGM + (cfg ^ ((pb & 3) << 1))] = make_double2(0.0, 0.0);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// After this thread's copies have landed: D[b][m] *= c_b(m) on its share
// (<m|a_q a_l|psi> = sqrt((u_q+1)(u_l+1)) psi_j for q < l, sqrt((u_q+1)(u_q+2)) psi_j for q = l).
template <int M, int kParts>
__device__ __forceinline__ void gemm_scale(const double *sq, double2 *D, const int (&u)[M], int cfg, int part)
{
    double r1[M], r2[M];   // sqrt(u_t + 1), sqrt((u_t + 1)(u_t + 2))
#pragma unroll
    for (int t = 0; t < M; ++t) {
        r1[t] = sq[u[t] + 1];
        r2[t] = r1[t] * sq[u[t] + 2];
    }
#pragma unroll
    for (int q = 0; q < M; ++q)
#pragma unroll
        for (int l = q; l < M; ++l) {
            const int pb = pair_index(q, l, M);
            if (pb % kParts == part) {
                const double c = (q == l) ? r2[q] : r1[q] * r1[l];
                double2 &d = D[pb * kGM + (cfg ^ ((pb & 3) << 1))];
                d.x *= c;
                d.y *= c;
            }
        }
}

// The factors c_b(m) of this thread's configuration into Cs, from the table
// ct (ct[x * nu + y] = sqrt(x+1) sqrt(y+1), ct[nu * nu + x] = sqrt(x+1) sqrt(x+2),
// the products the scaling would form): shared-memory loads and stores only.
template <int M>
__device__ __forceinline__ void gemm_coeffs(const double *ct, int nu, double *Cs, const int (&u)[M], int cfg)
{
#pragma unroll
    for (int q = 0; q < M; ++q)
#pragma unroll
        for (int l = q; l < M; ++l) {
            const int pb = pair_index(q, l, M);
            Cs[pb * kGM + (cfg ^ ((pb & 3) << 2))] = (q == l) ? ct[nu * nu + u[q]] : ct[u[q] * nu + u[l]];
        }
}

// One tile's product on the FP64 tensor cores (m16n8k4) and the E stores
// (warp-level): configurations m0 + 16 mg + (0 .. 15), pair tiles [T0, T1) (8 a each).
// With CS, D holds the bare gathered psi_j and Cs[b][m ^ ((b & 3) << 2)] the
// factor c_b(m); each lane scales its two A entries before the MMAs.
template <int M, int T0, int T1, bool CS>
__device__ __forceinline__ void gemm_tile16(const double2 *Hs, const double2 *D, const double *Cs,
                                            double2 *__restrict__ E, size_t stride, uint32_t nc2, uint32_t m0,
                                            int mg, int lane)
{
    using G = GemmShape<M>;
    constexpr int P = G::P, PK = G::PK, HS = G::HS, NT = T1 - T0;
    const int qr = lane >> 2, qc = lane & 3;
    const int mr0 = 16 * mg + qr, mr1 = mr0 + 8;  // this lane's two configurations within the tile
    // complex product in three real products: t1 = Dr Hr, t2 = Di Hi,
    // t3 = (Dr + Di)(Hr + Hi); Er = t1 - t2, Ei = t3 - t1 - t2
    double t1[NT][4], t2[NT][4], t3[NT][4];
#pragma unroll
    for (int t = 0; t < NT; ++t)
#pragma unroll
        for (int i = 0; i < 4; ++i) t1[t][i] = t2[t][i] = t3[t][i] = 0.0;
#pragma unroll 2
    for (int k0 = 0; k0 < PK; k0 += 4) {
        const int b = k0 + qc;
        const int sw = (b & 3) << 1;
        double2 d0 = D[b * kGM + (mr0 ^ sw)], d1 = D[b * kGM + (mr1 ^ sw)];
        if constexpr (CS) {
            const int cw = (b & 3) << 2;
            const double c0 = Cs[b * kGM + (mr0 ^ cw)], c1 = Cs[b * kGM + (mr1 ^ cw)];
            d0.x *= c0;
            d0.y *= c0;
            d1.x *= c1;
            d1.y *= c1;
        }
        const double s0 = d0.x + d0.y, s1 = d1.x + d1.y;
        double2 h[NT];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const int a = 8 * (T0 + t) + qr;
            h[t] = Hs[a * HS + (b ^ ((a & 1) << 2))];
        }
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            dmma16(t1[t], d0.x, d1.x, h[t].x);
            dmma16(t2[t], d0.y, d1.y, h[t].y);
            dmma16(t3[t], s0, s1, h[t].x + h[t].y);
        }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const uint32_t mo = m0 + (r ? mr1 : mr0);
        if (mo < nc2) {
#pragma unroll
            for (int t = 0; t < NT; ++t)
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int a = 8 * (T0 + t) + 2 * qc + i;
                    const int c = 2 * r + i;
                    if (a < P)
                        __stcs(E + a * stride + mo, make_double2(t1[t][c] - t2[t][c], t3[t][c] - t1[t][c] - t2[t][c]));
                }
        }
    }
}

template <int M>
__device__ __forceinline__ void gemm_load_h(const double2 *__restrict__ H, double2 *Hs, int nthreads)
{
    using G = GemmShape<M>;
    for (int x = threadIdx.x; x < G::PA * G::HS; x += nthreads) {
        const int a = x / G::HS, c = x % G::HS;
        const int b = c ^ ((a & 1) << 2);                          // logical column stored at c
        Hs[x] = (a < G::P && b < G::P) ? H[a * G::P + b] : make_double2(0.0, 0.0);
    }
}

// One block of 8 warps alternates gather and product on one D buffer (warp w:
// configurations 16 (w & 3) .. + 15, first or second half of the pair tiles);
// two blocks per SM (M <= 10) overlap one's gathers with the other's MMAs.
// Used when two D buffers do not fit shared memory.
template <int M>
__global__ void __launch_bounds__(kTG, M <= 10 ? 2 : 1)
    k_pair_annihilate_gemm(Space sp, SpaceTables tb, const double2 *__restrict__ H,
                           const double2 *__restrict__ psi, double2 *__restrict__ E, uint32_t ntiles)
{
    using G = GemmShape<M>;
    constexpr int P = G::P, PA = G::PA, PK = G::PK, HS = G::HS;
    constexpr int kParts = kTG / kGM;
    static_assert(kTG == 256 && kGM == 64, "8 warps: 4 groups of 16 configurations x 2 halves of the pair tiles");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *Hs = reinterpret_cast<double2 *>(smem_raw);          // PA x HS
    double2 *D = Hs + PA * HS;                                    // PK x kGM
    double *sq = reinterpret_cast<double *>(D + PK * kGM);
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);
    load_tables(sp, tb, W, sq);
    gemm_load_h<M>(H, Hs, kTG);
    for (int x = P * kGM + threadIdx.x; x < PK * kGM; x += kTG) D[x] = make_double2(0.0, 0.0);
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cfg = threadIdx.x % kGM, part = threadIdx.x / kGM;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int u[M];
        gemm_gather<M, kParts>(sp, tb, W, psi, D, tile * kGM + cfg, cfg, part, u);
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        gemm_scale<M, kParts>(sq, D, u, cfg, part);
        __syncthreads();
        constexpr int NH = (G::NT + 1) / 2;
        const int mg = warp & 3;
        if (warp < 4)
            gemm_tile16<M, 0, NH, false>(Hs, D, nullptr, E, sp.nc2, (uint32_t)sp.nc2, tile * kGM, mg, lane);
        else if constexpr (NH < G::NT)
            gemm_tile16<M, NH, G::NT, false>(Hs, D, nullptr, E, sp.nc2, (uint32_t)sp.nc2, tile * kGM, mg, lane);
        __syncthreads();   // every warp done with D before the next gather
    }
}

// Warp-specialised form (one block per SM): warps 0-15 run the products with
// m16n8k4 MMAs (warp w takes configurations 16 (w & 3) .. 16 (w & 3) + 15 of
// the tile and quarter w >> 2 of the pair tiles, so each SM sub-partition runs
// all pair tiles of one group of 16 configurations), warps 16-19 gather the next
// tiles into the other NS - 1 D buffers meanwhile: one thread per configuration
// (decoded once, all P gathers and scalings), warps 16-17 for the even tiles of
// the block, 18-19 for the odd ones. Tile i of a block uses buffer i % NS.
// Hand-over by mbarriers:
//   full[b]  : the 64 gather threads of the tile arrive after scaling buffer b; product
//              warps wait on its phase (tile i: parity (i / NS) & 1);
//   empty[b] : lane 0 of each of the 16 product warps arrives after reading
//              buffer b when a later tile of this block reuses it (i + NS < its
//              tile count); the gatherers wait on it (tile i >= NS: parity
//              (i / NS - 1) & 1) before overwriting.
// Product warps never wait for one another. Every wait is bounded: after
// kWaitCycles the thread records the timeout in the status word and returns
// (with no copies of its own in flight), so a stuck pipeline ends the kernel
// with an error instead of hanging.
constexpr int kTW = 2 * kTG + 2 * kGM;   // threads per block, warp-specialised form
template <int M, int NS, bool CS>
__global__ void __launch_bounds__(kTW, 1)
    k_pair_annihilate_gemm_ws(Space sp, SpaceTables tb, const double2 *__restrict__ H,
                              const double2 *__restrict__ psi, double2 *__restrict__ E, uint32_t ntiles,
                              int *status, long long wait_cycles, int test_stall)
{
    const long long limit = wait_cycles > 0 ? wait_cycles : kWaitCycles;
    using G = GemmShape<M>;
    constexpr int P = G::P, PA = G::PA, PK = G::PK, HS = G::HS;
    constexpr int kProdThreads = 2 * kTG;
    constexpr int kGroups = (kTW - kProdThreads) / kGM;   // gather groups of kGM threads
    static_assert(kTG == 256 && kGM == 64 && kGroups == 2, "16 product warps, 2 x 2 gather warps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *Hs = reinterpret_cast<double2 *>(smem_raw);          // PA x HS
    double2 *Dbuf = Hs + PA * HS;                                 // NS x (PK x kGM)
    double *Cbuf = reinterpret_cast<double *>(Dbuf + NS * PK * kGM);      // NS x (PK x kGM) when CS
    uint64_t *full = reinterpret_cast<uint64_t *>(Cbuf + (CS ? NS * PK * kGM : 0));  // NS
    uint64_t *empty = full + NS;                                           // NS
    double *sq = reinterpret_cast<double *>(empty + NS);
    const int nu = sp.N - 1;                                       // occupations 0 .. N-2
    double *ct = sq + sp.wstride;                                  // nu * nu + nu when CS
    uint32_t *W = reinterpret_cast<uint32_t *>(ct + (CS ? nu * nu + nu : 0));
    load_tables(sp, tb, W, sq);
    gemm_load_h<M>(H, Hs, kTW);
    for (int x = P * kGM + threadIdx.x; x < PK * kGM; x += kTW)
#pragma unroll
        for (int b = 0; b < NS; ++b) {
            Dbuf[b * PK * kGM + x] = make_double2(0.0, 0.0);
            if (CS) Cbuf[b * PK * kGM + x] = 0.0;
        }
    if (CS) {
        __syncthreads();   // sq loaded
        for (int x = threadIdx.x; x < nu * nu + nu; x += kTW)
            ct[x] = x < nu * nu ? sq[x / nu + 1] * sq[x % nu + 1] : sq[x - nu * nu + 1] * sq[x - nu * nu + 2];
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int b = 0; b < NS; ++b) {
            mbar_init(full + b, kGM);
            mbar_init(empty + b, kProdThreads / 32);
        }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ntb = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    if (warp >= kProdThreads / 32) {
        const int g = threadIdx.x - kProdThreads;
        const int cfg = g % kGM, grp = g / kGM;
        for (uint32_t i = grp; i < ntb; i += kGroups) {
            const int buf = i % NS;
            double2 *D = Dbuf + buf * PK * kGM;
            if (test_stall) return;   // test switch: deliver nothing, no copies issued
            if (i >= NS && !mbar_wait(empty + buf, (i / NS - 1) & 1, limit)) {
                atomicExch(status, 1);
                return;
            }
            int u[M];
            gemm_gather<M, 1>(sp, tb, W, psi, D, (blockIdx.x + i * gridDim.x) * kGM + cfg, cfg, 0, u);
            if constexpr (CS) gemm_coeffs<M>(ct, nu, Cbuf + buf * PK * kGM, u, cfg);
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            if constexpr (!CS) gemm_scale<M, 1>(sq, D, u, cfg, 0);
            mbar_arrive(full + buf);
        }
    } else {
        constexpr int NT = G::NT;
        constexpr int T1 = (NT + 3) / 4, T2 = (2 * NT + 3) / 4, T3 = (3 * NT + 3) / 4;
        const int mg = warp & 3, ap = warp >> 2;
        for (uint32_t i = 0; i < ntb; ++i) {
            const int buf = i % NS;
            if (!mbar_wait(full + buf, (i / NS) & 1, limit)) {
                if (lane == 0) atomicExch(status, 1);
                return;
            }
            const uint32_t m0 = (blockIdx.x + i * gridDim.x) * kGM;
            const double2 *D = Dbuf + buf * PK * kGM;
            const double *Cs = Cbuf + buf * PK * kGM;
            const uint32_t n2 = (uint32_t)sp.nc2;
            if (ap == 0) {
                gemm_tile16<M, 0, T1, CS>(Hs, D, Cs, E, sp.nc2, n2, m0, mg, lane);
            } else if (ap == 1) {
                if constexpr (T1 < T2) gemm_tile16<M, T1, T2, CS>(Hs, D, Cs, E, sp.nc2, n2, m0, mg, lane);
            } else if (ap == 2) {
                if constexpr (T2 < T3) gemm_tile16<M, T2, T3, CS>(Hs, D, Cs, E, sp.nc2, n2, m0, mg, lane);
            } else {
                if constexpr (T3 < NT) gemm_tile16<M, T3, NT, CS>(Hs, D, Cs, E, sp.nc2, n2, m0, mg, lane);
            }
            __syncwarp();
            if (lane == 0 && i + NS < ntb) mbar_arrive(empty + buf);
        }
    }
}

// ---------------------------------------------------------------------------
// kernel 1, block-sparse form: the same E, one pair-matrix block at a time.
// Each thread keeps, per orbital t, X[t] = B0[t]-B1[t], Y[t] = B1[t]-B2[t]
// (so index(m + e_q + e_l) = nc - 1 - (X[q] + Y[l] + B2[M-1]), q <= l) and the
// creation factors a[t] = sqrt(u_t+1), c[t] = sqrt((u_t+1)(u_t+2)) in shared
// memory columns it alone touches; a block's <= kBlockCols gathers are issued
// back to back into registers, then its rows are contracted and stored.
// ---------------------------------------------------------------------------
constexpr int kT1b = 128;

template <int M>
__global__ void __launch_bounds__(kT1b) k_pair_annihilate_blocks(Space sp, SpaceTables tb,
                                                                 BlockOp bo,
                                                                 const double2 *__restrict__ psi,
                                                                 double2 *__restrict__ E)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // layout: prog (bo.bytes, 16-aligned) | a,c doubles [M][kT1b] | X,Y uint32 [M][kT1b] | sq | W
    int *prog = reinterpret_cast<int *>(smem_raw);
    const int pbytes = (bo.bytes + 15) & ~15;
    double *fa = reinterpret_cast<double *>(smem_raw + pbytes);
    double *fc = fa + M * kT1b;
    uint32_t *X = reinterpret_cast<uint32_t *>(fc + M * kT1b);
    uint32_t *Y = X + M * kT1b;
    double *sq = reinterpret_cast<double *>(Y + M * kT1b);
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);
    for (int x = threadIdx.x; x < bo.bytes / 4; x += blockDim.x) prog[x] = bo.prog[x];
    load_tables(sp, tb, W, sq);
    __syncthreads();

    const int t = threadIdx.x;
    const uint32_t m = blockIdx.x * kT1b + t;
    if (m >= sp.nc2) return;
    const int ws = sp.wstride;
    {
        int u[M], Q[M];
        occupations<M>(tb.occ2, tb.occ_bits, m, sp.N - 2, sp.nc2, W, ws, u, Q);
        uint32_t B0[M], B1[M], B2[M];
        prefix_table<M>(Q, 0, W, ws, B0);
        prefix_table<M>(Q, 1, W, ws, B1);
        prefix_table<M>(Q, 2, W, ws, B2);
        const uint32_t base = sp.nc - 1u - B2[M - 1];
#pragma unroll
        for (int o = 0; o < M; ++o) {
            X[o * kT1b + t] = base - (B0[o] - B1[o]);   // base - X - Y = index
            Y[o * kT1b + t] = B1[o] - B2[o];
            fa[o * kT1b + t] = sq[u[o] + 1];
            fc[o * kT1b + t] = sq[u[o] + 1] * sq[u[o] + 2];
        }
    }
    const int nblocks = prog[0], ncols = prog[1], nrows = prog[2];
    const int *hdr = prog + 4;
    const int *cols = hdr + 5 * nblocks;
    const int *rows = cols + ncols;
    const double2 *vals = reinterpret_cast<const double2 *>(
        reinterpret_cast<const unsigned char *>(prog) + (((4 + 5 * nblocks + ncols + nrows) * 4 + 15) & ~15));
    const size_t stride = sp.nc2;
    for (int b = 0; b < nblocks; ++b) {
        const int cb = hdr[5 * b], nc_b = hdr[5 * b + 1], rb = hdr[5 * b + 2], nr_b = hdr[5 * b + 3],
                  vb = hdr[5 * b + 4];
        double2 d[kBlockCols];
#pragma unroll
        for (int c = 0; c < kBlockCols; ++c) {
            if (c < nc_b) {
                const int ql = cols[cb + c], q = ql & 0xff, l = ql >> 8;
                const uint32_t j = X[q * kT1b + t] - Y[l * kT1b + t];
                const double f = (q == l) ? fc[q * kT1b + t] : fa[q * kT1b + t] * fa[l * kT1b + t];
                const double2 x = __ldg(psi + j);
                d[c] = make_double2(f * x.x, f * x.y);
            }
        }
        for (int r = 0; r < nr_b; ++r) {
            double2 e = make_double2(0.0, 0.0);
            const double2 *hv = vals + vb + r * nc_b;
#pragma unroll
            for (int c = 0; c < kBlockCols; ++c)
                if (c < nc_b) cfma(e, hv[c], d[c]);
            E[(size_t)rows[rb + r] * stride + m] = e;
        }
    }
}

// ---------------------------------------------------------------------------
// kernel 1, momentum-block form. With plane-wave orbitals a translation-
// invariant interaction conserves momentum, so Ht[a][b] vanishes unless the
// pairs a = (k,s) and b = (q,l) have the same total k + s = q + l = K: Ht is
// block diagonal with one block per K = 0 .. 2M-2 (pairs q = max(0,K-M+1) ..
// K/2, l = K - q). The block layout is then a compile-time function of M,
// so every index, gather and block value offset below is a constant after
// unrolling: the prefix tables and gathered values stay in registers.
// hblk holds the blocks' dense values in that order (row-major per block).
// ---------------------------------------------------------------------------
// PARAM: hblk points at a __grid_constant__ kernel parameter; every block value
// index below is a compile-time constant, so its reads are constant-bank
// operands. Otherwise hblk is global memory and the values are staged in
// shared memory.
// How E entries are stored and loaded. The two-kernel path streams E through
// (evict-first stores and loads: it does not fit in L2); the fused path keeps
// it in L2 between its producer and consumer tiles.
enum : int {
    kEStoreStream = 0,     // st.global.cs
    kEStorePlain = 1,      // st.global (write-back)
    kEStoreKeep = 2,       // st.global with an L2 evict_last cache policy
};
enum : int {
    kELoadStream = 0,      // ld.global.cs
    kELoadDrop = 1,        // ld.global.cg with an L2 evict_first cache policy
    kELoadL2 = 2,          // ld.global.cg
};

__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}

template <int EST>
__device__ __forceinline__ void store_e(double2 *a, double2 v, uint64_t pol)
{
    if constexpr (EST == kEStoreStream) {
        __stcs(a, v);
    } else if constexpr (EST == kEStorePlain) {
        *a = v;
    } else {
        asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;\n" ::"l"(a), "d"(v.x), "d"(v.y),
                     "l"(pol)
                     : "memory");
    }
}

template <int ELD>
__device__ __forceinline__ double2 load_e(const double2 *a, uint64_t pol)
{
    if constexpr (ELD == kELoadStream) {
        return __ldcs(a);
    } else if constexpr (ELD == kELoadL2) {
        return __ldcg(a);
    } else {
        double2 v;
        asm volatile("ld.global.cg.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;\n"
                     : "=d"(v.x), "=d"(v.y)
                     : "l"(a), "l"(pol));
        return v;
    }
}

// One (N-2)-configuration m of kernel 1, momentum-block form: gathers its
// values <m|a_q a_l|psi> block by block and writes E[a][m] for every pair a.
// W, sq: the space's tables (shared memory); hv: the block values.
// ESTN / ESTF: store flavour of the pairs a = (k <= s) with s < FAR (near) and
// s >= FAR (far).
template <int M, int ESTN, int ESTF = ESTN, int FAR = M>
__device__ __forceinline__ void annihilate_momentum_row(const Space &sp, const SpaceTables &tb,
                                                        const uint32_t *W, const double *sq,
                                                        const double2 *__restrict__ hv,
                                                        const double2 *__restrict__ psi,
                                                        double2 *__restrict__ E, uint32_t m, uint64_t pol)
{
    const int ws = sp.wstride;
    int u[M], Q[M];
    occupations<M>(tb.occ2, tb.occ_bits, m, sp.N - 2, sp.nc2, W, ws, u, Q);
    uint32_t B0[M], B1[M], B2[M];
    prefix_table<M>(Q, 0, W, ws, B0);
    prefix_table<M>(Q, 1, W, ws, B1);
    prefix_table<M>(Q, 2, W, ws, B2);
    double fa[M];
    uint32_t Xa[M], Ya[M];   // index(m + e_q + e_l) = Xa[q] - Ya[l]  (q <= l)
    {
        const uint32_t base = sp.nc - 1u - B2[M - 1];
#pragma unroll
        for (int o = 0; o < M; ++o) {
            fa[o] = sq[u[o] + 1];
            Xa[o] = base - (B0[o] - B1[o]);
            Ya[o] = B1[o] - B2[o];
        }
    }
    const size_t stride = sp.nc2;
    constexpr int NB = M / 2 + 1;   // widest block
    int off = 0;
#pragma unroll
    for (int K = 0; K <= 2 * M - 2; ++K) {
        const int qlo = K - (M - 1) > 0 ? K - (M - 1) : 0, qhi = K / 2, n = qhi - qlo + 1;
        double2 d[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if (c < n) {
                const int q = qlo + c, l = K - q;
                const uint32_t j = Xa[q] - Ya[l];
                const double f = fa[q] * ((q == l) ? sq[u[q] + 2] : fa[l]);
                const double2 x = __ldg(psi + j);
                d[c] = make_double2(f * x.x, f * x.y);
            }
#pragma unroll
        for (int r = 0; r < NB; ++r)
            if (r < n) {
                double2 e = make_double2(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < NB; ++c)
                    if (c < n) cfma(e, hv[off + r * n + c], d[c]);
                double2 *dst = E + (size_t)pair_index(qlo + r, K - qlo - r, M) * stride + m;
                if (K - qlo - r >= FAR)
                    store_e<ESTF>(dst, e, pol);
                else
                    store_e<ESTN>(dst, e, pol);
            }
        off += n * n;
    }
}

// Configurations m0 + block * kT2 + t below m1 (the whole space: 0, nc2).
template <int M, bool PARAM = false>
__device__ __forceinline__ void annihilate_momentum_body(const Space &sp, const SpaceTables &tb,
                                                         const double2 *__restrict__ hblk, int nh,
                                                         const double2 *__restrict__ psi,
                                                         double2 *__restrict__ E, uint32_t block,
                                                         uint32_t m0 = 0, uint32_t m1 = 0xffffffffu)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *hs = reinterpret_cast<double2 *>(smem_raw);          // nh (staged form only)
    double *sq = reinterpret_cast<double *>(hs + (PARAM ? 0 : nh)); // wstride
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);  // (M-1) x wstride
    load_tables(sp, tb, W, sq);
    if (!PARAM)
        for (int x = threadIdx.x; x < nh; x += blockDim.x) hs[x] = hblk[x];
    const double2 *hv = PARAM ? hblk : hs;
    __syncthreads();

    const uint32_t m = m0 + block * kT2 + threadIdx.x;
    if (m >= sp.nc2 || m >= m1) return;
    annihilate_momentum_row<M, kEStoreStream>(sp, tb, W, sq, hv, psi, E, m, 0);
}

template <int M>
__global__ void __launch_bounds__(kT2, 3) k_pair_annihilate_momentum(Space sp, SpaceTables tb,
                                                                  const double2 *__restrict__ hblk,
                                                                  int nh,
                                                                  const double2 *__restrict__ psi,
                                                                  double2 *__restrict__ E, uint32_t m0,
                                                                  uint32_t m1)
{
    annihilate_momentum_body<M>(sp, tb, hblk, nh, psi, E, blockIdx.x, m0, m1);
}

// Number of momentum-block values for M orbitals (sum over K of block size squared).
template <int M>
constexpr int mom_values()
{
    int s = 0;
    for (int K = 0; K <= 2 * M - 2; ++K) {
        const int qlo = K - (M - 1) > 0 ? K - (M - 1) : 0, n = K / 2 - qlo + 1;
        s += n * n;
    }
    return s;
}

template <int M>
struct MomBlocks {
    double2 v[mom_values<M>()];
};

template <int M>
__global__ void __launch_bounds__(kT2, 3) k_pair_annihilate_momentum_p(Space sp, SpaceTables tb,
                                                                    const __grid_constant__ MomBlocks<M> hp,
                                                                    const double2 *__restrict__ psi,
                                                                    double2 *__restrict__ E, uint32_t m0,
                                                                    uint32_t m1)
{
    annihilate_momentum_body<M, true>(sp, tb, hp.v, mom_values<M>(), psi, E, blockIdx.x, m0, m1);
}

// ---------------------------------------------------------------------------
// kernel 2: out[i] = (sum_k Ho[k][k] v_k) psi[i] + sum_a c_a(v) E[a][index(v - pair a)]
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kT2, 4) k_pair_create(Space sp, SpaceTables tb, PairOp op,
                                                     const double2 *__restrict__ psi,
                                                     const double2 *__restrict__ E,
                                                     double2 *__restrict__ out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *hd = reinterpret_cast<double2 *>(smem_raw);          // M
    double *sq = reinterpret_cast<double *>(hd + M);              // wstride
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);  // (M-1) x wstride
    load_tables(sp, tb, W, sq);
    if (threadIdx.x < M) hd[threadIdx.x] = op.hdiag[threadIdx.x];
    __syncthreads();

    const uint32_t i = blockIdx.x * kT2 + threadIdx.x;
    if (i >= sp.nc) return;
    const int ws = sp.wstride;

    int v[M], P[M];
    occupations<M>(tb.occ, tb.occ_bits, i, sp.N, sp.nc, W, ws, v, P);

    double2 h1 = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < M; ++k) {
        h1.x += hd[k].x * v[k];
        h1.y += hd[k].y * v[k];
    }
    double2 acc = cmul(h1, psi[i]);

    if (sp.N >= 2) {
        // index(v - e_k - e_s) = Xr[k] - Yr[s] (k <= s) with
        // Xr[k] = nc2-1 - Am2[M-1] - (A0[k] - Am1[k]),  Yr[s] = Am1[s] - Am2[s]
        uint32_t Xr[M], Yr[M];
        double r1[M];   // sqrt(v_k): zero for an empty orbital, so empty pairs get weight 0
        {
            uint32_t A0[M], Am1[M], Am2[M];
            prefix_table<M>(P, 0, W, ws, A0);
            prefix_table<M>(P, -1, W, ws, Am1);
            prefix_table<M>(P, -2, W, ws, Am2);
            const uint32_t base = sp.nc2 - 1u - Am2[M - 1];
#pragma unroll
            for (int o = 0; o < M; ++o) {
                Xr[o] = base - (A0[o] - Am1[o]);
                Yr[o] = Am1[o] - Am2[o];
                r1[o] = sq[v[o]];
            }
        }
        const size_t stride = sp.nc2;
        // Branch-free: an empty pair has weight 0 and reads E[a][0] (one cached
        // line per pair), so the loads issue without waiting on occupancy tests.
#pragma unroll
        for (int k = 0; k < M; ++k)
#pragma unroll
            for (int s = k; s < M; ++s) {
                const double c = (s == k) ? r1[k] * sq[v[k] >= 1 ? v[k] - 1 : 0] : r1[k] * r1[s];
                const uint32_t mm = c != 0.0 ? Xr[k] - Yr[s] : 0u;
                const double2 e = __ldg(E + pair_index(k, s, M) * stride + mm);
                acc.x = fma(c, e.x, acc.x);
                acc.y = fma(c, e.y, acc.y);
            }
    }
    out[i] = acc;
}

// Kernel 2, shared-table form (default): the per-row tables (Xr, Yr, sqrt v_k
// and v_k - 1) live in shared-memory columns that only their thread touches,
// so the pair loop needs few registers (no spills) and occupancy is set by
// shared memory (17 bytes per orbital and row). Measured at N=16, M=10:
// 0.183 ms with the E gathers issued in groups of 8 (0.198 ms consumed one by
// one, 0.186 ms in groups of 16), against 0.238 ms with two double tables, 0.248 ms for the register
// form, 0.216 ms keeping only occupation bytes (square roots looked up per
// pair), 0.21 ms forcing five blocks per SM (spills); staging each block's
// contiguous E ranges in shared memory with TMA bulk copies (0.73 ms) or
// prefetching them into L2 (0.28 ms) was slower still.
// One N-configuration i of kernel 2, shared-table form: row tables into this
// thread's shared-memory columns (r1, Xr, Yr, vb), then the gathers. row:
// i is a row to compute (out[i - row0]). ELDN / ELDF: how E is loaded for the
// pairs (k <= s) with s < FAR and s >= FAR. STREAM_OUT: write out with an
// evict-first store.
template <int M, int ELDN, int ELDF = ELDN, int FAR = M, bool STREAM_OUT = false>
__device__ __forceinline__ void create_row(const Space &sp, const SpaceTables &tb, const uint32_t *W,
                                           const double *sq, const double2 *hd,
                                           const double2 *__restrict__ psi, const double2 *E,
                                           double2 *__restrict__ out, uint32_t i, bool row, uint32_t row0,
                                           double *r1, uint32_t *Xr, uint32_t *Yr, unsigned char *vb,
                                           uint64_t pol)
{
    const int t = threadIdx.x;
    const int ws = sp.wstride;
    double2 acc;
    {
        int v[M], P[M];
        occupations<M>(tb.occ, tb.occ_bits, row ? i : (tb.occ ? row0 : 0u), sp.N, sp.nc, W, ws, v, P);
        double2 h1 = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            h1.x += hd[k].x * v[k];
            h1.y += hd[k].y * v[k];
        }
        acc = row ? cmul(h1, psi[i]) : make_double2(0.0, 0.0);
        if (sp.N < 2) {
            if (row) out[i - row0] = acc;
            return;
        }
        uint32_t A0[M], Am1[M], Am2[M];
        prefix_table<M>(P, 0, W, ws, A0);
        prefix_table<M>(P, -1, W, ws, Am1);
        prefix_table<M>(P, -2, W, ws, Am2);
        const uint32_t base = sp.nc2 - 1u - Am2[M - 1];
#pragma unroll
        for (int o = 0; o < M; ++o) {
            Xr[o * kTC + t] = base - (A0[o] - Am1[o]);
            Yr[o * kTC + t] = Am1[o] - Am2[o];
            r1[o * kTC + t] = row ? sq[v[o]] : 0.0;
            vb[o * kTC + t] = (unsigned char)(v[o] >= 1 ? v[o] - 1 : 0);
        }
    }
    const size_t stride = sp.nc2;
    if (!row) return;
    // pairs p = pair_index(k, s) in order, in groups of kCreateBatch: all loads
    // of a group are issued before any is consumed (E is read exactly once:
    // streaming loads), so each thread keeps a group of gathers in flight
    constexpr int NPR = M * (M + 1) / 2;
#pragma unroll
    for (int p0 = 0; p0 < NPR; p0 += kCreateBatch) {
        double cc[kCreateBatch];
        double2 ee[kCreateBatch];
#pragma unroll
        for (int j = 0; j < kCreateBatch; ++j) {
            const int p = p0 + j;
            if (p < NPR) {
                int k = 0, rem = p;   // (k, s) of pair p, resolved at compile time
#pragma unroll
                for (int kk = 0; kk < M; ++kk)
                    if (rem >= M - kk && k == kk) {
                        rem -= M - kk;
                        k = kk + 1;
                    }
                const int s = k + rem;
                const double c = r1[k * kTC + t] * ((s == k) ? sq[vb[k * kTC + t]] : r1[s * kTC + t]);
                const uint32_t mm = Xr[k * kTC + t] - Yr[s * kTC + t];
                cc[j] = c;
                // empty pairs (c = 0: their index is meaningless) load nothing
                const double2 *src = E + (size_t)p * stride + mm;
                ee[j] = c == 0.0     ? make_double2(0.0, 0.0)
                        : s >= FAR   ? load_e<ELDF>(src, pol)
                                     : load_e<ELDN>(src, pol);
            }
        }
#pragma unroll
        for (int j = 0; j < kCreateBatch; ++j)
            if (p0 + j < NPR) {
                acc.x = fma(cc[j], ee[j].x, acc.x);
                acc.y = fma(cc[j], ee[j].y, acc.y);
            }
    }
    if constexpr (STREAM_OUT)
        __stcs(out + (i - row0), acc);
    else
        out[i - row0] = acc;
}

// Kernel 2, shared-table form (default): the per-row tables (Xr, Yr, sqrt v_k
// and v_k - 1) live in shared-memory columns that only their thread touches,
// so the pair loop needs few registers (no spills) and occupancy is set by
// shared memory (17 bytes per orbital and row). Measured at N=16, M=10:
// 0.183 ms with the E gathers issued in groups of 8 (0.198 ms consumed one by
// one, 0.186 ms in groups of 16), against 0.238 ms with two double tables, 0.248 ms for the register
// form, 0.216 ms keeping only occupation bytes (square roots looked up per
// pair), 0.21 ms forcing five blocks per SM (spills); staging each block's
// contiguous E ranges in shared memory with TMA bulk copies (0.73 ms) or
// prefetching them into L2 (0.28 ms) was slower still.
template <int M>
__device__ __forceinline__ void create_smem_body(const Space &sp, const SpaceTables &tb,
                                                 const double2 *__restrict__ hdiag,
                                                 const double2 *__restrict__ psi,
                                                 const double2 *__restrict__ E,
                                                 double2 *__restrict__ out, uint32_t block,
                                                 uint32_t row0, uint32_t row1)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *r1 = reinterpret_cast<double *>(smem_raw);             // M x kTC
    uint32_t *Xr = reinterpret_cast<uint32_t *>(r1 + M * kTC);     // M x kTC
    uint32_t *Yr = Xr + M * kTC;                                   // M x kTC
    unsigned char *vb = reinterpret_cast<unsigned char *>(Yr + M * kTC);   // M x kTC
    double2 *hd = reinterpret_cast<double2 *>(vb + ((M * kTC + 15) & ~15)); // M
    double *sq = reinterpret_cast<double *>(hd + M);               // wstride
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);   // (M-1) x wstride
    load_tables(sp, tb, W, sq);
    if (threadIdx.x < M) hd[threadIdx.x] = hdiag[threadIdx.x];
    __syncthreads();

    const uint32_t i = row0 + block * kTC + threadIdx.x;   // rows [row0, row1) -> out[i - row0]
    create_row<M, kELoadStream>(sp, tb, W, sq, hd, psi, E, out, i, i < row1, row0, r1, Xr, Yr, vb, 0);
}

template <int M>
__global__ void __launch_bounds__(kTC, 4) k_pair_create_smem(Space sp, SpaceTables tb, PairOp op,
                                                          const double2 *__restrict__ psi,
                                                          const double2 *__restrict__ E,
                                                          double2 *__restrict__ out, uint32_t row0,
                                                          uint32_t row1)
{
    // blocks run from the top rows down: their E entries (images near the end of
    // each E row) are the ones kernel 1 wrote last, some still in L2
    create_smem_body<M>(sp, tb, op.hdiag, psi, E, out, gridDim.x - 1 - blockIdx.x, row0, row1);
}

// ---------------------------------------------------------------------------
// Direct H.psi, momentum-block form: no intermediate. Written out per row,
//   (H2 psi)(v) = sum_{a occupied in v} c_a(v) sum_{b in block(a)} Ht[a][b] c_b(v - a) psi[v - a + b],
// the pair-space product with nothing stored between its two halves: every
// term gathers straight from psi, which stays in L2 (32.7 MB at N=16, M=10),
// so HBM carries only psi, out and the occupation table (about 82 MB against
// the 1.5 GB of the two-kernel form with its P x NC(N-2,M) intermediate E).
// Within a momentum block a = (k, s) and b = (q, l) have k + s = q + l, so
// for b != a the orbitals q, l differ from k, s and one of two orders holds,
// q < k <= s < l or k < q <= l < s. The prefix counts of v - a + b then move
// by +1 on [q, k) and -1 on [s, l) (or -1 on [k, q) and +1 on [l, s)); with
// per-row tables F[t] = sum_{i<t} W_i(P_i + 1) - W_i(P_i) and G (the same
// with P_i - 1) the target index splits into a part of a and a part of b:
// with YA(p) = F[q] - G[l], YB(p) = F[l] - G[q] for a pair p = (q, l),
//   q < k:  (base - YA(a)) + YA(b)
//   q > k:  (base - YB(a)) + YB(b),
// two numbers per pair, formed once per block, so a term costs one addition
// for its index. c_b(v - a) = sqrt((v_q+1)(v_l+1)) (sqrt((v_q+1)(v_q+2)) for
// q = l) depends on v alone; the diagonal term b = a reads psi[v] with
// c_a(v)^2. Square-root products come from a table sqrt(x) sqrt(y) in shared
// memory; c_a(v) = 0 tells that a is not in v. The gathers of R creation
// pairs of a block are issued together. REAL: the block values are real (any
// real translation-invariant interaction), so a term is a real coefficient
// times a complex gather -- two multiply-adds instead of four, the same
// values. SMEM_D: the tables F, G sit in shared-memory columns of their
// thread instead of registers. The kernel is bound on the SM (L1 data pipe,
// then instruction issue), not by HBM. The products of creation pairs that a
// row does not hold run predicated with c_a = 0: skipping them by branches,
// divergent or warp-uniform, measured slower, because the straight-line code
// keeps the gathers of every block in flight.
// ---------------------------------------------------------------------------
// Shared memory of a direct block: hd[M] | sqrt(x) sqrt(y) [ws x ws] |
// W [(M-1) x ws] | (SMEM_D) F, G [M x kTC] each.
template <int M>
constexpr size_t direct_smem(int ws, bool smem_d)
{
    return sizeof(double2) * M + sizeof(double) * ws * ws + sizeof(uint32_t) * (M - 1) * ws +
           (smem_d ? 2 * sizeof(uint32_t) * M * kTC : 0);
}

template <int M>
__device__ __forceinline__ void direct_tables(int ws, const uint32_t *gW, const double *gsq, const double2 *hdiag,
                                              double2 *hd, double *sqp, uint32_t *W)
{
    for (int x = threadIdx.x; x < (M - 1) * ws; x += blockDim.x) W[x] = gW[x];
    for (int x = threadIdx.x; x < ws * ws; x += blockDim.x) sqp[x] = gsq[x / ws] * gsq[x % ws];
    if (threadIdx.x < M) hd[threadIdx.x] = hdiag[threadIdx.x];
}

// Row i of H.psi in the direct form into *dst; hv(x) is block value x.
template <int M, bool REAL, int R, bool SMEM_D, class HV>
__device__ __forceinline__ void direct_row(const Space &sp, const uint64_t *occ, int occ_bits, const uint32_t *W,
                                           const double *sqp, const double2 *hd, uint32_t *FS, uint32_t *GS,
                                           const HV &hv, const double2 *__restrict__ psi, double2 *dst, uint32_t i)
{
    const int ws = sp.wstride;
    int vv[M], P[M];
    occupations<M>(occ, occ_bits, i, sp.N, sp.nc, W, ws, vv, P);
    const double2 x0 = __ldg(psi + i);
    double2 acc;
    {
        double2 h1 = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            h1.x += hd[k].x * vv[k];
            h1.y += hd[k].y * vv[k];
        }
        acc = cmul(h1, x0);
    }
    // F[t] = sum_{i<t} W_i(P_i + 1) - W_i(P_i), G[t] the same with P_i - 1
    uint32_t F[M], G[M], s0 = 0;
    F[0] = G[0] = 0;
#pragma unroll
    for (int t = 1; t < M; ++t) {
        const uint32_t w0 = W[(t - 1) * ws + P[t - 1]];
        s0 += w0;
        F[t] = F[t - 1] + (W[(t - 1) * ws + P[t - 1] + 1] - w0);
        G[t] = G[t - 1] + (wlook(W, ws, t - 1, P[t - 1] - 1) - w0);
    }
    const uint32_t base = sp.nc - 1u - s0;
    if constexpr (SMEM_D) {
#pragma unroll
        for (int t = 0; t < M; ++t) {
            FS[t * kTC + threadIdx.x] = F[t];
            GS[t * kTC + threadIdx.x] = G[t];
        }
    }
    auto f = [&](int t) -> uint32_t { return SMEM_D ? FS[t * kTC + threadIdx.x] : F[t]; };
    auto g = [&](int t) -> uint32_t { return SMEM_D ? GS[t * kTC + threadIdx.x] : G[t]; };
    // (occupations packed into one 64-bit word, unpacked at every use,
    // measured 2 % slower than the array)
    auto v = [&](int o) -> int { return vv[o]; };
    constexpr int NB = M / 2 + 1;
    int off = 0;
#pragma unroll
    for (int K = 0; K <= 2 * M - 2; ++K) {
        const int qlo = K - (M - 1) > 0 ? K - (M - 1) : 0, qhi = K / 2, n = qhi - qlo + 1;
        if (n == 1) {   // a single pair: only its diagonal term
            const int k = qlo, s = K - k;
            const double ca2 = k == s ? (double)(v(k) * (v(k) - 1)) : (double)(v(k) * v(s));
            const double2 h = hv(off);
            cfma(acc, make_double2(h.x * ca2, h.y * ca2), x0);
            off += 1;
            continue;
        }
        // per pair p = (q, l) of the block: its index parts YA = F[q] - G[l],
        // YB = F[l] - G[q] (as a creation pair its X = base - Y) and its
        // creation factor c_p(v - a) = sqrt(v_q + 1) sqrt(v_l + 1)
        uint32_t YA[NB], YB[NB];
        double cb[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if (c < n) {
                const int q = qlo + c, l = K - q;
                YA[c] = f(q) - g(l);
                YB[c] = f(l) - g(q);
                cb[c] = sqp[(v(q) + 1) * ws + (q == l ? v(q) + 2 : v(l) + 1)];
            }
#pragma unroll
        for (int r0 = 0; r0 < NB; r0 += R)
            if (r0 < n) {
                double2 gv[R][NB];
                double ca[R];
#pragma unroll
                for (int rr = 0; rr < R; ++rr) {
                    const int r = r0 + rr;
                    if (r < n) {
                        const int k = qlo + r, s = K - k;
                        // c_a(v) = sqrt(v_k) sqrt(v_s) (sqrt(v_k) sqrt(v_k - 1) for k = s): zero iff a is not in v
                        ca[rr] = sqp[v(k) * ws + (k == s ? max(v(k) - 1, 0) : v(s))];
                        const bool occ = ca[rr] != 0.0;
                        const uint32_t XA = base - YA[r], XB = base - YB[r];
#pragma unroll
                        for (int c = 0; c < NB; ++c)
                            if (c < n && c != r) {
                                const uint32_t j = c < r ? XA + YA[c] : XB + YB[c];
                                gv[rr][c] = occ ? __ldg(psi + j) : make_double2(0.0, 0.0);
                            }
                    }
                }
#pragma unroll
                for (int rr = 0; rr < R; ++rr) {
                    const int r = r0 + rr;
                    if (r < n) {
                        double2 e = make_double2(0.0, 0.0);
#pragma unroll
                        for (int c = 0; c < NB; ++c)
                            if (c < n) {
                                const double2 h = hv(off + r * n + c);
                                const double w = c == r ? ca[rr] : cb[c];
                                const double2 y = c == r ? x0 : gv[rr][c];
                                if constexpr (REAL) {
                                    const double t = h.x * w;
                                    e.x = fma(t, y.x, e.x);
                                    e.y = fma(t, y.y, e.y);
                                } else {
                                    cfma(e, make_double2(h.x * w, h.y * w), y);
                                }
                            }
                        acc.x = fma(ca[rr], e.x, acc.x);
                        acc.y = fma(ca[rr], e.y, acc.y);
                    }
                }
            }
        off += n * n;
    }
    *dst = acc;
}

template <int M, bool REAL, int R, bool SMEM_D>
__global__ void __launch_bounds__(kTC, 3)
    k_hpsi_direct(Space sp, SpaceTables tb, const __grid_constant__ MomBlocks<M> hp,
                  const double2 *__restrict__ hdiag, const double2 *__restrict__ psi, double2 *__restrict__ out,
                  uint32_t row0, uint32_t row1)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ws = sp.wstride;
    double2 *hd = reinterpret_cast<double2 *>(smem_raw);
    double *sqp = reinterpret_cast<double *>(hd + M);
    uint32_t *W = reinterpret_cast<uint32_t *>(sqp + ws * ws);
    uint32_t *FS = W + (M - 1) * ws, *GS = FS + M * kTC;
    direct_tables<M>(ws, tb.W, tb.sq, hdiag, hd, sqp, W);
    __syncthreads();
    const uint32_t i = row0 + blockIdx.x * kTC + threadIdx.x;   // rows [row0, row1) -> out[i - row0]
    if (i >= row1) return;
    direct_row<M, REAL, R, SMEM_D>(sp, tb.occ, tb.occ_bits, W, sqp, hd, FS, GS,
                                   [&](int x) -> double2 { return hp.v[x]; }, psi, out + (i - row0), i);
}

template <int M, bool REAL>
cudaError_t launch_direct(const Space &sp, const SpaceTables &tb, const MomBlocks<M> &hp, const double2 *hdiag,
                          const double2 *psi, double2 *out, cudaStream_t st, uint32_t row0, uint32_t row1)
{
    // two creation pairs' gathers in flight, the index tables in shared-memory
    // columns (the fastest of the forms measured at N=16 and N=20, M=10)
    constexpr int R = 2;
    constexpr bool SMEM_D = true;
    const size_t smem = direct_smem<M>(sp.wstride, SMEM_D);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k_hpsi_direct<M, REAL, R, SMEM_D>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const unsigned grid = (row1 - row0 + kTC - 1) / kTC;
    k_hpsi_direct<M, REAL, R, SMEM_D><<<grid, kTC, smem, st>>>(sp, tb, hp, hdiag, psi, out, row0, row1);
    return cudaGetLastError();
}

template <int M>
cudaError_t direct_apply_m(const Space &sp, const SpaceTables &tb, const PairOp &op, const double2 *psi,
                           double2 *out, cudaStream_t st, uint32_t row0, uint32_t row1)
{
    if (row1 <= row0) return cudaSuccess;
    MomBlocks<M> hp;
    bool real = true;
    for (int x = 0; x < mom_values<M>(); ++x) {
        hp.v[x] = op.hblk_host[x];
        real = real && hp.v[x].y == 0.0;
    }
    if (real) return launch_direct<M, true>(sp, tb, hp, op.hdiag, psi, out, st, row0, row1);
    return launch_direct<M, false>(sp, tb, hp, op.hdiag, psi, out, st, row0, row1);
}

}  // namespace

// Number of momentum-block values for M orbitals, at run time.
static int mom_count(int M)
{
    int s = 0;
    for (int K = 0; K <= 2 * M - 2; ++K) {
        const int qlo = K - (M - 1) > 0 ? K - (M - 1) : 0, n = K / 2 - qlo + 1;
        s += n * n;
    }
    return s;
}

int hpsi_form(const Space &sp, const PairOp &op)
{
    if (sp.N < 2 || sp.M < 2 || !op.hblk_host || op.nhblk != mom_count(sp.M)) return kFormTwo;
    // N < 64 bounds the square-root product table, (N + 3)^2 doubles of shared memory
    if (op.direct && sp.N < 64 && op.create_form == 0 && (op.direct != 2 || sp.M <= kDirectAutoMaxM))
        return kFormDirect;
    if (op.fused.order && op.create_form == 0) return kFormFused;
    return kFormTwo;
}

namespace {

// ---------------------------------------------------------------------------
// Fused H.psi, momentum-block form (FusedPlan in kernels.h). The two-kernel
// path writes all of E (P x NC(N-2,M) complex, 719 MB at N=16, M=10) to HBM
// and reads it back. Here one persistent grid walks kernel 1's tiles and
// kernel 2's tiles in one order: consumer tile c (rows in index order) comes
// right after the producer tiles up to need[c]. For a fixed pair a the map
// v -> v - e_k - e_s keeps the index order, so the E columns a consumer reads
// lie just behind the producer front, and the E alive between its write and
// its read stays in L2 (peak 53 MB, mean 19 MB at N=16, M=10, against 126 MB).
//
// Hand-over: producer tiles are counted in groups of kFusedGroup; a producer
// block stores its E, then (thread 0, after a barrier and a device-scope
// fence) adds one to its group's counter. A consumer's thread 0 waits until
// every group up to need[c] / kFusedGroup is complete (acquire loads; it
// remembers the groups it has seen complete, so each group is checked by a
// block at most until it is), then the block reads. Items are handed out in
// order from a ticket counter and producers never wait, so every tile a
// consumer waits for belongs to a running block: the waits end. A block grabs
// its next ticket early -- at the start of a producer tile, or once a
// consumer's wait is over -- never while it may still wait, so a held ticket
// always belongs to a block that will reach it. The waits are bounded all the
// same (about two seconds): one that runs out sets the abort word and the
// status word and its block skips the tile (out is then invalid; the next
// synchronising call reports MCPI_ERR_TIMEOUT); every later consumer sees the
// abort word and skips at once. test_stall (a test switch) keeps the
// producers from counting, so that the waits run out. The last block to leave
// zeroes the counters for the next call (or graph replay).
//
// Each consumer row does exactly the arithmetic of kernel 2 on exactly the
// values kernel 1 writes, so the fused result is bitwise the two-kernel one.
//
// Which pairs stay in L2. A pair a = (k, s) that includes the top orbital
// (s = M-1) moves a configuration a whole slab of the index order (the top
// occupation is the most significant digit), so its E column is read about
// a slab after it is written: at N=16, M=10 those 10 of the 55 pairs account
// for 15 of the 19 MB mean live window. They are written and read as in the
// two-kernel form (evict-first streaming, through HBM); the other pairs are
// stored with an evict-last and loaded with an evict-first L2 policy (mean
// live window 4 MB).
//
// Measured (N=16, M=10, Lieb, B200): 0.365 ms per H.psi at a lead of 192
// tiles against 0.300 ms for the two kernels. DRAM traffic falls from about
// 1.5 GB to 1.1 GB -- the reads of E mostly hit L2, but every dirty E line is
// still written back when L2 evicts it -- while the kernel is bound by
// latency and barriers at three blocks per SM (80 registers; four blocks
// spill and run at 0.41 ms). So the two-kernel form stays the default.
// ---------------------------------------------------------------------------
// control words, each on its own 128-byte line (FusedPlan::ctl)
enum : int { kFzTicket = 0, kFzExited = 32, kFzAbort = 64 };

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *a)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(a) : "memory");
    return v;
}

__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned *a)
{
    return *reinterpret_cast<const volatile unsigned *>(a);
}

__device__ __forceinline__ int fused_item(const FusedPlan &fz, unsigned k)
{
    return k < (unsigned)fz.nitems ? fz.order[k] : INT_MIN;
}

template <int M>
__global__ void __launch_bounds__(kTC, 3)
    k_hpsi_fused(Space sp, SpaceTables tb, const __grid_constant__ MomBlocks<M> hp,
                 const double2 *__restrict__ hdiag, const double2 *__restrict__ psi, double2 *E,
                 double2 *__restrict__ out, FusedPlan fz, int *status, long long wait_cycles, int test_stall)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *r1 = reinterpret_cast<double *>(smem_raw);             // M x kTC
    uint32_t *Xr = reinterpret_cast<uint32_t *>(r1 + M * kTC);     // M x kTC
    uint32_t *Yr = Xr + M * kTC;                                   // M x kTC
    unsigned char *vb = reinterpret_cast<unsigned char *>(Yr + M * kTC);   // M x kTC
    double2 *hd = reinterpret_cast<double2 *>(vb + ((M * kTC + 15) & ~15)); // M
    double *sq = reinterpret_cast<double *>(hd + M);               // wstride
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);   // (M-1) x wstride
    __shared__ int s_item[2];
    __shared__ int s_ok;
    const int t = threadIdx.x;
    load_tables(sp, tb, W, sq);
    if (t < M) hd[t] = hdiag[t];
    if (t == 0) s_item[0] = fused_item(fz, atomicAdd(fz.ctl + kFzTicket, 1u));
    __syncthreads();

    const long long limit = wait_cycles > 0 ? wait_cycles : kWaitCycles;
    const int ngroups = (fz.np + kFusedGroup - 1) / kFusedGroup;
    const uint64_t pst = l2_policy_evict_last(), pld = l2_policy_evict_first();
    int known = 0;   // (thread 0) producer groups below this are known to be complete

    for (int it = 0;; ++it) {
        const int item = s_item[it & 1];
        if (item == INT_MIN) break;
        unsigned ticket = 0;   // (thread 0) the next item's ticket, taken early, used at the end
        if (item >= 0) {
            // producer: kernel 1 on configurations [item * 256, item * 256 + 256)
            if (t == 0) ticket = atomicAdd(fz.ctl + kFzTicket, 1u);
            const uint32_t m = (uint32_t)item * kFusedTile + t;
            if (m < sp.nc2)
                annihilate_momentum_row<M, kEStoreKeep, kEStoreStream, M - 1>(sp, tb, W, sq, hp.v, psi, E, m, pst);
            __syncthreads();
            if (t == 0) {
                if (!test_stall) {
                    __threadfence();
                    atomicAdd(fz.count + item / kFusedGroup, 1u);
                }
                s_item[(it + 1) & 1] = fused_item(fz, ticket);
            }
        } else {
            // consumer: kernel 2 on rows [c * 256, c * 256 + 256)
            const int c = -1 - item;
            if (t == 0) {
                const int gneed = fz.need[c] / kFusedGroup;
                int ok = 1;
                const long long t0 = clock64();
                while (known <= gneed) {
                    const unsigned full = known + 1 < ngroups ? kFusedGroup : fz.np - known * kFusedGroup;
                    if (ld_acquire_u32(fz.count + known) == full) {
                        ++known;
                        continue;
                    }
                    if (ld_volatile_u32(fz.ctl + kFzAbort)) {
                        ok = 0;
                        break;
                    }
                    if (clock64() - t0 > limit) {
                        atomicExch(fz.ctl + kFzAbort, 1u);
                        if (status) atomicExch(status, 1);
                        ok = 0;
                        break;
                    }
                    __nanosleep(200);
                }
                __threadfence();
                s_ok = ok;
                // the wait is over: this block reaches its next item in bounded time
                ticket = atomicAdd(fz.ctl + kFzTicket, 1u);
            }
            __syncthreads();
            if (s_ok) {
                const uint32_t i = (uint32_t)c * kFusedTile + t;
                create_row<M, kELoadDrop, kELoadStream, M - 1, true>(sp, tb, W, sq, hd, psi, E, out, i, i < sp.nc,
                                                                      0u, r1, Xr, Yr, vb, pld);
            }
            if (t == 0) s_item[(it + 1) & 1] = fused_item(fz, ticket);
        }
        __syncthreads();   // the next item is visible; s_ok is free again
    }
    // the last block out zeroes the counters for the next call
    __shared__ int s_last;
    if (t == 0) {
        __threadfence();
        s_last = atomicAdd(fz.ctl + kFzExited, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        for (int g = t; g < ngroups; g += blockDim.x) fz.count[g] = 0u;
        if (t == 0) {
            fz.ctl[kFzTicket] = 0u;
            fz.ctl[kFzAbort] = 0u;
            fz.ctl[kFzExited] = 0u;
        }
        __threadfence();
    }
}

// need[c]: the highest producer tile that consumer tile c reads. The largest
// E column a row v reads is that of its two lowest particles (removing them
// changes only the least significant occupations of the index order).
template <int M>
__global__ void __launch_bounds__(kFusedTile) k_fused_need(Space sp, SpaceTables tb, int *need)
{
    extern __shared__ uint32_t Wd[];   // (M-1) x wstride
    __shared__ uint32_t s_max[kFusedTile / 32];
    const int ws = sp.wstride;
    for (int x = threadIdx.x; x < (M - 1) * ws; x += blockDim.x) Wd[x] = tb.W[x];
    __syncthreads();
    const uint32_t i = blockIdx.x * kFusedTile + threadIdx.x;
    uint32_t mx = 0;
    if (i < sp.nc) {
        int v[M], P[M];
        occupations<M>(tb.occ, tb.occ_bits, i, sp.N, sp.nc, Wd, ws, v, P);
        int k0 = 0;
        while (k0 < M - 1 && v[k0] == 0) ++k0;
        int k1 = k0;
        if (v[k0] < 2) {
            k1 = k0 + 1;
            while (k1 < M - 1 && v[k1] == 0) ++k1;
        }
        uint32_t A0[M], Am1[M], Am2[M];
        prefix_table<M>(P, 0, Wd, ws, A0);
        prefix_table<M>(P, -1, Wd, ws, Am1);
        prefix_table<M>(P, -2, Wd, ws, Am2);
        mx = idx_remove2(sp.nc2, A0, Am1, Am2, k0, k1, M);
    }
    for (int o = 16; o; o >>= 1) {
        const uint32_t y = __shfl_down_sync(0xffffffffu, mx, o);
        mx = y > mx ? y : mx;
    }
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kFusedTile / 32; ++w) mx = s_max[w] > mx ? s_max[w] : mx;
        need[blockIdx.x] = (int)(mx / kFusedTile);
    }
}

template <int M>
cudaError_t fused_apply_m(const Space &sp, const SpaceTables &tb, const PairOp &op, const double2 *psi,
                          double2 *E, double2 *out, cudaStream_t st)
{
    const size_t tab = sizeof(double) * sp.wstride + sizeof(uint32_t) * (M - 1) * sp.wstride;
    const size_t sm = (sizeof(double) + 2 * sizeof(uint32_t)) * M * kTC + ((M * kTC + 15) & ~15) +
                      sizeof(double2) * M + tab;
    if (sm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_hpsi_fused<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
    }
    MomBlocks<M> hp;
    for (int x = 0; x < mom_values<M>(); ++x) hp.v[x] = op.hblk_host[x];
    k_hpsi_fused<M><<<op.fused.grid, kTC, sm, st>>>(sp, tb, hp, op.hdiag, psi, E, out, op.fused, op.status,
                                                   op.wait_cycles, op.test_stall);
    return cudaGetLastError();
}

template <int M>
cudaError_t fused_config_m(const Space &sp, int *grid, size_t *smem)
{
    const size_t tab = sizeof(double) * sp.wstride + sizeof(uint32_t) * (M - 1) * sp.wstride;
    const size_t sm = (sizeof(double) + 2 * sizeof(uint32_t)) * M * kTC + ((M * kTC + 15) & ~15) +
                      sizeof(double2) * M + tab;
    const void *fn = (const void *)k_hpsi_fused<M>;
    cudaError_t e = cudaSuccess;
    if (sm > 48 * 1024 &&
        (e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) != cudaSuccess)
        return e;
    int dev = 0, sms = 0, per = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kTC, sm)) != cudaSuccess) return e;
    *grid = sms * (per > 0 ? per : 1);
    *smem = sm;
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Batched H.psi: one launch applies H to the current Lanczos vector of every
// member of a batch with the same M. A block's (member, block-in-member) pair
// comes from a work table, so members of any size share the grid; members
// whose Lanczos has stopped skip their blocks.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kT2, 3) k_batch_annihilate(const BatchMember *__restrict__ mem,
                                                          const int2 *__restrict__ work, int vec)
{
    const int2 w = work[blockIdx.x];
    const BatchMember &b = mem[w.x];
    if (*b.done) return;
    annihilate_momentum_body<M>(b.sp, SpaceTables{b.W, b.sq, b.occ, b.occ_bits, b.occ2}, b.hblk, b.nh,
                                b.lvec + (size_t)vec * b.sp.nc, b.E, (uint32_t)w.y);
}

template <int M>
__global__ void __launch_bounds__(kTC, 4) k_batch_create(const BatchMember *__restrict__ mem,
                                                      const int2 *__restrict__ work, int vec)
{
    const int2 w = work[blockIdx.x];
    const BatchMember &b = mem[w.x];
    if (*b.done) return;
    create_smem_body<M>(b.sp, SpaceTables{b.W, b.sq, b.occ, b.occ_bits, b.occ2}, b.hdiag, b.lvec + (size_t)vec * b.sp.nc, b.E,
                        b.r, (uint32_t)w.y, 0u, b.sp.nc);
}

// The direct form for a batch: one launch, blocks of kTC rows of any member
// (the creation work table), each block staging its member's block values in
// shared memory (members differ, so they cannot be a kernel parameter).
template <int M, bool REAL>
__global__ void __launch_bounds__(kTC, 3) k_batch_direct(const BatchMember *__restrict__ mem,
                                                      const int2 *__restrict__ work, int vec)
{
    const int2 w = work[blockIdx.x];
    const BatchMember &b = mem[w.x];
    if (*b.done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ws = b.sp.wstride;
    double2 *hv = reinterpret_cast<double2 *>(smem_raw);            // mom_values<M>()
    double2 *hd = hv + mom_values<M>();
    double *sqp = reinterpret_cast<double *>(hd + M);
    uint32_t *W = reinterpret_cast<uint32_t *>(sqp + ws * ws);
    uint32_t *FS = W + (M - 1) * ws, *GS = FS + M * kTC;
    for (int x = threadIdx.x; x < mom_values<M>(); x += blockDim.x) hv[x] = b.hblk[x];
    direct_tables<M>(ws, b.W, b.sq, b.hdiag, hd, sqp, W);
    __syncthreads();
    const uint32_t i = (uint32_t)w.y * kTC + threadIdx.x;
    if (i >= b.sp.nc) return;
    direct_row<M, REAL, 2, true>(b.sp, b.occ, b.occ_bits, W, sqp, hd, FS, GS,
                                 [&](int x) -> double2 { return hv[x]; }, b.lvec + (size_t)vec * b.sp.nc, b.r + i, i);
}

// Real block values of up to CAP members of one M, passed as a kernel
// parameter (at most 30 KB of the 32 KB a launch takes): every block reads its
// member's values through the constant bank, as the single-space kernel does,
// instead of from shared memory.
template <int M>
struct BatchVals {
    static constexpr int NV = mom_values<M>();
    static constexpr int CAP = (30 * 1024) / (8 * NV + 4) < 64 ? (30 * 1024) / (8 * NV + 4) : 64;
    double v[CAP][NV];
    int member[CAP];
};

template <int M>
__global__ void __launch_bounds__(kTC, 3) k_batch_direct_p(const BatchMember *__restrict__ mem,
                                                        const int2 *__restrict__ work, int vec,
                                                        const __grid_constant__ BatchVals<M> bv)
{
    const int2 w = work[blockIdx.x];   // (slot in bv, block of the member's rows)
    const int slot = w.x;
    const BatchMember &b = mem[bv.member[slot]];
    if (*b.done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ws = b.sp.wstride;
    double2 *hd = reinterpret_cast<double2 *>(smem_raw);
    double *sqp = reinterpret_cast<double *>(hd + M);
    uint32_t *W = reinterpret_cast<uint32_t *>(sqp + ws * ws);
    uint32_t *FS = W + (M - 1) * ws, *GS = FS + M * kTC;
    direct_tables<M>(ws, b.W, b.sq, b.hdiag, hd, sqp, W);
    __syncthreads();
    const uint32_t i = (uint32_t)w.y * kTC + threadIdx.x;
    if (i >= b.sp.nc) return;
    direct_row<M, true, 2, true>(b.sp, b.occ, b.occ_bits, W, sqp, hd, FS, GS,
                                 [&](int x) -> double2 { return make_double2(bv.v[slot][x], 0.0); },
                                 b.lvec + (size_t)vec * b.sp.nc, b.r + i, i);
}

template <int M>
cudaError_t batch_prepare_m(size_t smem1, size_t smem2, size_t smem3)
{
    cudaError_t e = cudaFuncSetAttribute(k_batch_annihilate<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem1);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_create<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_direct<M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem3);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_direct<M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem3);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_direct_p<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem3);
    return e;
}

template <int M>
cudaError_t batch_apply_m(int form, const BatchMember *mem, const int2 *work1, int n1, size_t smem1,
                          const int2 *work2, int n2, size_t smem2, int vec, cudaStream_t st)
{
    if (form == kBatchDirectReal) {
        if (n2) k_batch_direct<M, true><<<n2, kTC, smem2, st>>>(mem, work2, vec);
    } else if (form == kBatchDirectComplex) {
        if (n2) k_batch_direct<M, false><<<n2, kTC, smem2, st>>>(mem, work2, vec);
    } else {
        if (n1) k_batch_annihilate<M><<<n1, kT2, smem1, st>>>(mem, work1, vec);
        if (n2) k_batch_create<M><<<n2, kTC, smem2, st>>>(mem, work2, vec);
    }
    return cudaGetLastError();
}

// One particle: the configurations are the orbitals themselves (index(e_l) = l),
// so H psi = Ho psi.
__global__ void k_one_particle(int M, const double2 *__restrict__ hfull,
                               const double2 *__restrict__ psi, double2 *__restrict__ out)
{
    int k = threadIdx.x;
    if (k >= M) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int l = 0; l < M; ++l) cfma(acc, hfull[k * M + l], psi[l]);
    out[k] = acc;
}

template <int M>
cudaError_t apply_h_m(const Space &sp, const SpaceTables &tb, const PairOp &op, const BlockOp &bo,
                      const double2 *psi, double2 *E, double2 *out, int stages, cudaStream_t st,
                      uint32_t row0, uint32_t row1, uint32_t m0, uint32_t m1)
{
    constexpr int P = M * (M + 1) / 2;
    const size_t tab = sizeof(double) * sp.wstride + sizeof(uint32_t) * (M - 1) * sp.wstride;
    if constexpr (M >= 2) {
        if (stages == 3) {
            const int form = hpsi_form(sp, op);
            if (form == kFormDirect) return direct_apply_m<M>(sp, tb, op, psi, out, st, row0, row1);
            if (form == kFormFused && row0 == 0 && row1 == sp.nc)
                return fused_apply_m<M>(sp, tb, op, psi, E, out, st);
        }
    }
    if (sp.N >= 2 && (stages & 1) && op.hblk) {
        // only the configurations [m0, m1) (a row block's range; the whole space by default)
        if (m1 > sp.nc2) m1 = sp.nc2;
        const unsigned g1 = m1 > m0 ? (m1 - m0 + kT2 - 1) / kT2 : 0;
        if (g1 && op.hblk_host && op.nhblk == mom_values<M>()) {
            MomBlocks<M> hp;
            for (int x = 0; x < mom_values<M>(); ++x) hp.v[x] = op.hblk_host[x];
            k_pair_annihilate_momentum_p<M><<<g1, kT2, tab, st>>>(sp, tb, hp, psi, E, m0, m1);
        } else if (g1) {
            const size_t smm = sizeof(double2) * op.nhblk + tab;
            k_pair_annihilate_momentum<M><<<g1, kT2, smm, st>>>(sp, tb, op.hblk, op.nhblk, psi, E, m0, m1);
        }
    } else if (sp.N >= 2 && (stages & 1) && bo.prog) {
        const size_t smb = ((bo.bytes + 15) & ~15) + (2 * sizeof(double) + 2 * sizeof(uint32_t)) * M * kT1b + tab;
        if (smb > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(
                k_pair_annihilate_blocks<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb);
            if (e != cudaSuccess) return e;
        }
        const unsigned g1 = (sp.nc2 + kT1b - 1) / kT1b;
        k_pair_annihilate_blocks<M><<<g1, kT1b, smb, st>>>(sp, tb, bo, psi, E);
    } else if (sp.N >= 2 && (stages & 1) && op.hdense && P <= kGemmMaxP) {
        if constexpr (P <= kGemmMaxP) {
            using G = GemmShape<M>;
            int dev = 0, sms = 0, optin = 0;
            cudaError_t e;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
                return e;
            const uint32_t ntiles = (uint32_t)((sp.nc2 + kGM - 1) / kGM);
            const size_t nu = (size_t)sp.N - 1;
            const size_t cbytes = G::dbytes / 2;   // PK x kGM doubles
            const size_t smc2 = G::hbytes + 2 * (G::dbytes + cbytes) + 4 * sizeof(uint64_t) +
                                sizeof(double) * (nu * nu + nu) + tab;
            const size_t smw3 = G::hbytes + 3 * G::dbytes + 6 * sizeof(uint64_t) + tab;
            const size_t smw2 = G::hbytes + 2 * G::dbytes + 4 * sizeof(uint64_t) + tab;
            const unsigned gw = ntiles < (uint32_t)sms ? ntiles : (uint32_t)sms;
            if (smc2 <= (size_t)optin) {
                if ((e = cudaFuncSetAttribute(k_pair_annihilate_gemm_ws<M, 2, true>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc2)) != cudaSuccess)
                    return e;
                if (gw)
                    k_pair_annihilate_gemm_ws<M, 2, true>
                        <<<gw, kTW, smc2, st>>>(sp, tb, op.hdense, psi, E, ntiles, op.status,
                                                                         op.wait_cycles, op.test_stall);
            } else if (smw3 <= (size_t)optin) {
                if ((e = cudaFuncSetAttribute(k_pair_annihilate_gemm_ws<M, 3, false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw3)) != cudaSuccess)
                    return e;
                if (gw)
                    k_pair_annihilate_gemm_ws<M, 3, false>
                        <<<gw, kTW, smw3, st>>>(sp, tb, op.hdense, psi, E, ntiles, op.status,
                                                                         op.wait_cycles, op.test_stall);
            } else if (smw2 <= (size_t)optin) {
                if ((e = cudaFuncSetAttribute(k_pair_annihilate_gemm_ws<M, 2, false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw2)) != cudaSuccess)
                    return e;
                if (gw)
                    k_pair_annihilate_gemm_ws<M, 2, false>
                        <<<gw, kTW, smw2, st>>>(sp, tb, op.hdense, psi, E, ntiles, op.status,
                                                                         op.wait_cycles, op.test_stall);
            } else {
                const size_t smg = G::hbytes + G::dbytes + tab;
                if ((e = cudaFuncSetAttribute(k_pair_annihilate_gemm<M>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smg)) != cudaSuccess)
                    return e;
                const uint32_t per_sm = M <= 10 ? 2u : 1u;
                const unsigned g1 = ntiles < per_sm * sms ? ntiles : per_sm * sms;
                if (g1) k_pair_annihilate_gemm<M><<<g1, kTG, smg, st>>>(sp, tb, op.hdense, psi, E, ntiles);
            }
        }
    } else if (sp.N >= 2 && (stages & 1)) {
        const int st_nnz = op.nnz <= kCsrStaged ? op.nnz : 0;
        const size_t sm1 = sizeof(double2) * (P * kT1 + st_nnz) + tab + sizeof(int) * (P + 1 + st_nnz);
        if (sm1 > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(
                k_pair_annihilate<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
            if (e != cudaSuccess) return e;
        }
        const unsigned g1 = (sp.nc2 + kT1 - 1) / kT1;
        k_pair_annihilate<M><<<g1, kT1, sm1, st>>>(sp, tb, op, psi, E);
    }
    if ((stages & 2) && sp.N >= 2 && op.create_form == 0) {
        const size_t sm2 = (sizeof(double) + 2 * sizeof(uint32_t)) * M * kTC + ((M * kTC + 15) & ~15) +
                           sizeof(double2) * M + tab;
        if (sm2 > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(
                k_pair_create_smem<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
            if (e != cudaSuccess) return e;
        }
        const unsigned g2 = (row1 - row0 + kTC - 1) / kTC;
        if (g2) k_pair_create_smem<M><<<g2, kTC, sm2, st>>>(sp, tb, op, psi, E, out, row0, row1);
    } else if (stages & 2) {
        if (row0 != 0 || row1 != sp.nc) return cudaErrorInvalidValue;   // row ranges: shared-table form only
        const size_t sm2 = sizeof(double2) * M + tab;
        const unsigned g2 = (sp.nc + kT2 - 1) / kT2;
        k_pair_create<M><<<g2, kT2, sm2, st>>>(sp, tb, op, psi, E, out);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_batch_apply_h(int M, int form, const BatchMember *mem, const int2 *work1, int n1, size_t smem1,
                                 const int2 *work2, int n2, size_t smem2, int vec, cudaStream_t st)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: return batch_apply_m<m>(form, mem, work1, n1, smem1, work2, n2, smem2, vec, st);
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

int batch_chunk_members(int M)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: return BatchVals<m>::CAP;
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return 0;
    }
}

size_t batch_vals_bytes(int M)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: return sizeof(BatchVals<m>);
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return 0;
    }
}

namespace {
template <int M>
void fill_vals_m(void *vals, int slot, int member, const double2 *hblk_host)
{
    auto *bv = static_cast<BatchVals<M> *>(vals);
    bv->member[slot] = member;
    for (int x = 0; x < BatchVals<M>::NV; ++x) bv->v[slot][x] = hblk_host[x].x;
}
}  // namespace

void batch_fill_vals(int M, void *vals, int slot, int member, const double2 *hblk_host)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: fill_vals_m<m>(vals, slot, member, hblk_host); break;
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: break;
    }
}

cudaError_t launch_batch_direct_vals(int M, const BatchMember *mem, const int2 *work, int n, size_t smem, int vec,
                                     const void *vals, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    switch (M) {
#define MCPI_CASE(m) \
    case m:                                                                                              \
        k_batch_direct_p<m><<<n, kTC, smem, st>>>(mem, work, vec, *static_cast<const BatchVals<m> *>(vals)); \
        return cudaGetLastError();
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t batch_prepare(int M, size_t smem1, size_t smem2, size_t smem3)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: return batch_prepare_m<m>(smem1, smem2, smem3);
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

size_t batch_smem(int M, int N, int nh, int stage)
{
    const int ws = N + 3;
    const size_t tab = sizeof(double) * ws + sizeof(uint32_t) * (M - 1) * ws;
    if (stage == 1) return sizeof(double2) * nh + tab;
    if (stage == 3)   // the direct form: block values | hd | sqrt products | W | F, G
        return sizeof(double2) * (nh + M) + sizeof(double) * ws * ws + sizeof(uint32_t) * (M - 1) * ws +
               2 * sizeof(uint32_t) * M * kTC;
    return (sizeof(double) + 2 * sizeof(uint32_t)) * M * kTC + ((M * kTC + 15) & ~15) + sizeof(double2) * M +
           tab;
}

int batch_rows_per_block(int stage) { return stage == 1 ? kT2 : kTC; }

namespace {

// The (N-2)-configurations rows [r0, r1) read in kernel 2: every row reads
// index(v - e_k - e_s) for its occupied pairs, the largest from its two lowest
// particles and the smallest from its two highest (the top occupation is the
// most significant digit of the index order). out[0] = min, out[1] = max
// (initialised by the caller to UINT32_MAX and 0).
template <int M>
__global__ void __launch_bounds__(kFusedTile) k_rows_mrange(Space sp, SpaceTables tb, uint32_t r0, uint32_t r1,
                                                            uint32_t *out)
{
    extern __shared__ uint32_t Wr[];   // (M-1) x wstride
    const int ws = sp.wstride;
    for (int x = threadIdx.x; x < (M - 1) * ws; x += blockDim.x) Wr[x] = tb.W[x];
    __syncthreads();
    const uint32_t i = r0 + blockIdx.x * kFusedTile + threadIdx.x;
    uint32_t lo = 0xffffffffu, hi = 0u;
    if (i < r1) {
        int v[M], P[M];
        occupations<M>(tb.occ, tb.occ_bits, i, sp.N, sp.nc, Wr, ws, v, P);
        int k0 = 0;
        while (k0 < M - 1 && v[k0] == 0) ++k0;
        int k1 = k0;
        if (v[k0] < 2) {
            k1 = k0 + 1;
            while (k1 < M - 1 && v[k1] == 0) ++k1;
        }
        int s1 = M - 1;
        while (s1 > 0 && v[s1] == 0) --s1;
        int s0 = s1;
        if (v[s1] < 2) {
            s0 = s1 - 1;
            while (s0 > 0 && v[s0] == 0) --s0;
        }
        uint32_t A0[M], Am1[M], Am2[M];
        prefix_table<M>(P, 0, Wr, ws, A0);
        prefix_table<M>(P, -1, Wr, ws, Am1);
        prefix_table<M>(P, -2, Wr, ws, Am2);
        hi = idx_remove2(sp.nc2, A0, Am1, Am2, k0, k1, M);
        lo = idx_remove2(sp.nc2, A0, Am1, Am2, s0, s1, M);
    }
    for (int o = 16; o; o >>= 1) {
        const uint32_t a = __shfl_down_sync(0xffffffffu, lo, o), b = __shfl_down_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(out, lo);
        atomicMax(out + 1, hi);
    }
}

}  // namespace

cudaError_t launch_rows_mrange(const Space &sp, const SpaceTables &tb, uint32_t r0, uint32_t r1, uint32_t *out,
                               cudaStream_t st)
{
    if (sp.N < 2 || sp.M < 2 || r1 <= r0 || r1 > sp.nc) return cudaErrorInvalidValue;
    const uint32_t init[2] = {0xffffffffu, 0u};
    cudaError_t e = cudaMemcpyAsync(out, init, sizeof init, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    const unsigned g = (r1 - r0 + kFusedTile - 1) / kFusedTile;
    const size_t sm = sizeof(uint32_t) * (sp.M - 1) * sp.wstride;
    switch (sp.M) {
#define MCPI_CASE(m) \
    case m: k_rows_mrange<m><<<g, kFusedTile, sm, st>>>(sp, tb, r0, r1, out); return cudaGetLastError();
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fused_need(const Space &sp, const SpaceTables &tb, int *need, cudaStream_t st)
{
    if (sp.N < 2 || sp.M < 2) return cudaErrorInvalidValue;
    const unsigned g = (sp.nc + kFusedTile - 1) / kFusedTile;
    const size_t sm = sizeof(uint32_t) * (sp.M - 1) * sp.wstride;
    switch (sp.M) {
#define MCPI_CASE(m) \
    case m: k_fused_need<m><<<g, kFusedTile, sm, st>>>(sp, tb, need); return cudaGetLastError();
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t fused_config(const Space &sp, int *grid, size_t *smem)
{
    switch (sp.M) {
#define MCPI_CASE(m) \
    case m: return fused_config_m<m>(sp, grid, smem);
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_apply_h(const Space &sp, const SpaceTables &tb, const PairOp &op,
                           const BlockOp &bo, const double2 *psi, double2 *E, double2 *out,
                           cudaStream_t st, int stages, uint32_t row0, uint32_t row1, uint32_t m0,
                           uint32_t m1)
{
    if (row1 == 0xffffffffu) row1 = sp.nc;
    if (row0 > row1 || row1 > sp.nc) return cudaErrorInvalidValue;
    if (sp.N == 1) {
        if (row0 != 0 || row1 != sp.nc) return cudaErrorInvalidValue;
        if (stages & 2) k_one_particle<<<1, 32, 0, st>>>(sp.M, op.hfull, psi, out);
        return cudaGetLastError();
    }
    switch (sp.M) {
#define MCPI_CASE(m) \
    case m: return apply_h_m<m>(sp, tb, op, bo, psi, E, out, stages, st, row0, row1, m0, m1);
        MCPI_CASE(1) MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6)
        MCPI_CASE(7) MCPI_CASE(8) MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12)
        MCPI_CASE(13) MCPI_CASE(14) MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace mcpi
