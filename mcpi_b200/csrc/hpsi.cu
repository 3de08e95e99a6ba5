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

namespace mcpi {

namespace {

constexpr int kT1 = 64;    // threads (= (N-2)-configurations) per block, kernel 1
constexpr int kCsrStaged = 1024;   // pair-matrix nonzeros staged in shared memory
constexpr int kT2 = 256;   // threads per block, kernel 2 (register form) and kernel 1 (momentum form)
constexpr int kTC = 256;   // threads (= rows) per block, kernel 2 (shared-table form)

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
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
    decode<M>(m, sp.N - 2, sp.nc2, W, ws, u, Q);
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
// kernel 1, dense-product form for general pair matrices (P <= kGemmMaxP).
// A persistent block keeps Ht (P x P, zero-padded to PA = 8 * RA rows) in
// shared memory. Per tile of kGM (N-2)-configurations it gathers
// D[b][m] = c_b(m) psi[index(m + pair b)] into shared memory (kTG / kGM threads
// per configuration, cp.async), then forms E[a][m] = sum_b Ht[a][b] D[b][m] as a
// register-tiled complex FP64 product: warp w owns the rows a = w*RA .. w*RA+RA-1
// (Ht reads are warp-uniform broadcasts), lane owns the columns m = lane and
// lane + 32 (conflict-free 16-byte reads of D, coalesced evict-first stores of E).
// Per configuration: P gathers, 4 P^2 FP64 FMAs, P stores.
// ---------------------------------------------------------------------------
constexpr int kTG = 256;   // threads per block, dense-product form
constexpr int kGM = 64;    // (N-2)-configurations per tile

template <int M>
__global__ void __launch_bounds__(kTG, M <= 10 ? 2 : 1) k_pair_annihilate_gemm(Space sp, SpaceTables tb,
                                                                 const double2 *__restrict__ H,
                                                                 const double2 *__restrict__ psi,
                                                                 double2 *__restrict__ E, uint32_t ntiles)
{
    constexpr int P = M * (M + 1) / 2;
    constexpr int RA = (P + 7) / 8;
    constexpr int PA = 8 * RA;
    constexpr int kParts = kTG / kGM;
    static_assert(kTG == 256 && kGM == 64, "8 warps x RA rows, 2 columns per lane");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *Hs = reinterpret_cast<double2 *>(smem_raw);          // PA x P
    double2 *D = Hs + PA * P;                                     // P x kGM
    double *sq = reinterpret_cast<double *>(D + P * kGM);
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);
    load_tables(sp, tb, W, sq);
    for (int x = threadIdx.x; x < PA * P; x += kTG) Hs[x] = x < P * P ? H[x] : make_double2(0.0, 0.0);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cfg = threadIdx.x % kGM, part = threadIdx.x / kGM;
    const int ws = sp.wstride;
    const size_t stride = sp.nc2;
    const double2 *Hw = Hs + warp * RA * P;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t m0 = tile * kGM;
        const uint32_t m = m0 + cfg;
        __syncthreads();   // tables loaded (first tile) / previous tile's D consumed
        if (m < sp.nc2) {
            int u[M], Q[M];
            decode<M>(m, sp.N - 2, sp.nc2, W, ws, u, Q);
            uint32_t B0[M], B1[M], B2[M];
            prefix_table<M>(Q, 0, W, ws, B0);
            prefix_table<M>(Q, 1, W, ws, B1);
            prefix_table<M>(Q, 2, W, ws, B2);
#pragma unroll
            for (int q = 0; q < M; ++q)
#pragma unroll
                for (int l = q; l < M; ++l)
                    if (pair_index(q, l, M) % kParts == part) {
                        const uint32_t j = idx_add2(sp.nc, B0, B1, B2, q, l, M);
                        cp_async16(D + pair_index(q, l, M) * kGM + cfg, psi + j);
                    }
            cp_async_wait_all();
#pragma unroll
            for (int q = 0; q < M; ++q)
#pragma unroll
                for (int l = q; l < M; ++l)
                    if (pair_index(q, l, M) % kParts == part) {
                        const double c = (q == l) ? sq[u[q] + 1] * sq[u[q] + 2] : sq[u[q] + 1] * sq[u[l] + 1];
                        double2 &d = D[pair_index(q, l, M) * kGM + cfg];
                        d.x *= c;
                        d.y *= c;
                    }
        } else {
            for (int b = part; b < P; b += kParts) D[b * kGM + cfg] = make_double2(0.0, 0.0);
        }
        __syncthreads();

        double2 acc0[RA], acc1[RA];
#pragma unroll
        for (int i = 0; i < RA; ++i) acc0[i] = acc1[i] = make_double2(0.0, 0.0);
#pragma unroll 5
        for (int k = 0; k < P; ++k) {
            const double2 d0 = D[k * kGM + lane], d1 = D[k * kGM + lane + 32];
#pragma unroll
            for (int i = 0; i < RA; ++i) {
                const double2 h = Hw[i * P + k];
                cfma(acc0[i], h, d0);
                cfma(acc1[i], h, d1);
            }
        }
        const bool ok0 = m0 + lane < sp.nc2, ok1 = m0 + lane + 32 < sp.nc2;
#pragma unroll
        for (int i = 0; i < RA; ++i) {
            const int a = warp * RA + i;
            if (a < P) {
                if (ok0) __stcs(E + a * stride + m0 + lane, acc0[i]);
                if (ok1) __stcs(E + a * stride + m0 + lane + 32, acc1[i]);
            }
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
        decode<M>(m, sp.N - 2, sp.nc2, W, ws, u, Q);
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
template <int M>
__device__ __forceinline__ void annihilate_momentum_body(const Space &sp, const SpaceTables &tb,
                                                         const double2 *__restrict__ hblk, int nh,
                                                         const double2 *__restrict__ psi,
                                                         double2 *__restrict__ E, uint32_t block)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *hv = reinterpret_cast<double2 *>(smem_raw);          // nh
    double *sq = reinterpret_cast<double *>(hv + nh);             // wstride
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);  // (M-1) x wstride
    load_tables(sp, tb, W, sq);
    for (int x = threadIdx.x; x < nh; x += blockDim.x) hv[x] = hblk[x];
    __syncthreads();

    const uint32_t m = block * kT2 + threadIdx.x;
    if (m >= sp.nc2) return;
    const int ws = sp.wstride;
    int u[M], Q[M];
    decode<M>(m, sp.N - 2, sp.nc2, W, ws, u, Q);
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
                __stcs(E + (size_t)pair_index(qlo + r, K - qlo - r, M) * stride + m, e);
            }
        off += n * n;
    }
}

template <int M>
__global__ void __launch_bounds__(kT2, 3) k_pair_annihilate_momentum(Space sp, SpaceTables tb,
                                                                  const double2 *__restrict__ hblk,
                                                                  int nh,
                                                                  const double2 *__restrict__ psi,
                                                                  double2 *__restrict__ E)
{
    annihilate_momentum_body<M>(sp, tb, hblk, nh, psi, E, blockIdx.x);
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
    decode<M>(i, sp.N, sp.nc, W, ws, v, P);

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
// 0.198 ms, against 0.238 ms with two double tables, 0.248 ms for the register
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

    const int t = threadIdx.x;
    const uint32_t i = row0 + block * kTC + t;   // rows [row0, row1) -> out[i - row0]
    const bool row = i < row1;
    const int ws = sp.wstride;
    double2 acc;
    {
        int v[M], P[M];
        decode<M>(row ? i : 0u, sp.N, sp.nc, W, ws, v, P);
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
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int s = k; s < M; ++s) {
            const double c = r1[k * kTC + t] * ((s == k) ? sq[vb[k * kTC + t]] : r1[s * kTC + t]);
            const uint32_t mm = c != 0.0 ? Xr[k * kTC + t] - Yr[s * kTC + t] : 0u;
            const double2 e = __ldg(E + pair_index(k, s, M) * stride + mm);
            acc.x = fma(c, e.x, acc.x);
            acc.y = fma(c, e.y, acc.y);
        }
    out[i - row0] = acc;
}

template <int M>
__global__ void __launch_bounds__(kTC) k_pair_create_smem(Space sp, SpaceTables tb, PairOp op,
                                                          const double2 *__restrict__ psi,
                                                          const double2 *__restrict__ E,
                                                          double2 *__restrict__ out, uint32_t row0,
                                                          uint32_t row1)
{
    create_smem_body<M>(sp, tb, op.hdiag, psi, E, out, blockIdx.x, row0, row1);
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
    annihilate_momentum_body<M>(b.sp, SpaceTables{b.W, b.sq}, b.hblk, b.nh,
                                b.lvec + (size_t)vec * b.sp.nc, b.E, (uint32_t)w.y);
}

template <int M>
__global__ void __launch_bounds__(kTC) k_batch_create(const BatchMember *__restrict__ mem,
                                                      const int2 *__restrict__ work, int vec)
{
    const int2 w = work[blockIdx.x];
    const BatchMember &b = mem[w.x];
    if (*b.done) return;
    create_smem_body<M>(b.sp, SpaceTables{b.W, b.sq}, b.hdiag, b.lvec + (size_t)vec * b.sp.nc, b.E,
                        b.r, (uint32_t)w.y, 0u, b.sp.nc);
}

template <int M>
cudaError_t batch_prepare_m(size_t smem1, size_t smem2)
{
    cudaError_t e = cudaFuncSetAttribute(k_batch_annihilate<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem1);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_batch_create<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
    return e;
}

template <int M>
cudaError_t batch_apply_m(const BatchMember *mem, const int2 *work1, int n1, size_t smem1,
                          const int2 *work2, int n2, size_t smem2, int vec, cudaStream_t st)
{
    if (n1) k_batch_annihilate<M><<<n1, kT2, smem1, st>>>(mem, work1, vec);
    if (n2) k_batch_create<M><<<n2, kTC, smem2, st>>>(mem, work2, vec);
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
                      uint32_t row0, uint32_t row1)
{
    constexpr int P = M * (M + 1) / 2;
    const size_t tab = sizeof(double) * sp.wstride + sizeof(uint32_t) * (M - 1) * sp.wstride;
    if (sp.N >= 2 && (stages & 1) && op.hblk) {
        const size_t smm = sizeof(double2) * op.nhblk + tab;
        const unsigned g1 = (sp.nc2 + kT2 - 1) / kT2;
        k_pair_annihilate_momentum<M><<<g1, kT2, smm, st>>>(sp, tb, op.hblk, op.nhblk, psi, E);
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
            constexpr int PA = 8 * ((P + 7) / 8);
            const size_t smg = sizeof(double2) * (PA * P + P * kGM) + tab;
            cudaError_t e = cudaFuncSetAttribute(k_pair_annihilate_gemm<M>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smg);
            if (e != cudaSuccess) return e;
            int dev = 0, sms = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            const uint32_t ntiles = (uint32_t)((sp.nc2 + kGM - 1) / kGM);
            const unsigned g1 = ntiles < 2u * sms ? ntiles : 2u * sms;
            if (g1) k_pair_annihilate_gemm<M><<<g1, kTG, smg, st>>>(sp, tb, op.hdense, psi, E, ntiles);
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

cudaError_t launch_batch_apply_h(int M, const BatchMember *mem, const int2 *work1, int n1, size_t smem1,
                                 const int2 *work2, int n2, size_t smem2, int vec, cudaStream_t st)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: return batch_apply_m<m>(mem, work1, n1, smem1, work2, n2, smem2, vec, st);
        MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6) MCPI_CASE(7) MCPI_CASE(8)
        MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12) MCPI_CASE(13) MCPI_CASE(14)
        MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t batch_prepare(int M, size_t smem1, size_t smem2)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: return batch_prepare_m<m>(smem1, smem2);
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
    return (sizeof(double) + 2 * sizeof(uint32_t)) * M * kTC + ((M * kTC + 15) & ~15) + sizeof(double2) * M +
           tab;
}

int batch_rows_per_block(int stage) { return stage == 1 ? kT2 : kTC; }

cudaError_t launch_apply_h(const Space &sp, const SpaceTables &tb, const PairOp &op,
                           const BlockOp &bo, const double2 *psi, double2 *E, double2 *out,
                           cudaStream_t st, int stages, uint32_t row0, uint32_t row1)
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
    case m: return apply_h_m<m>(sp, tb, op, bo, psi, E, out, stages, st, row0, row1);
        MCPI_CASE(1) MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6)
        MCPI_CASE(7) MCPI_CASE(8) MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12)
        MCPI_CASE(13) MCPI_CASE(14) MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace mcpi
