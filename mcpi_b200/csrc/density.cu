// One- and two-body (transition) densities.
//
// Reference: onebodyMatrix.h:34-251 (OBrho*) and twobodyMatrix.h:38-1487
// (TBrho*) compute rho1[k][l] = <a+_k a_l> and rho2[k+sM+qM^2+lM^3] =
// <a+_k a+_s a_q a_l> for one state, reducing each unique index tuple over all
// nc rows (M^4/8 passes over psi for rho2) and filling the rest by symmetry.
//
// B200 formulation. Both are Gram matrices over a hole space:
//     rho1[k][l]        = sum_{m in N-1}  conj(<m|a_k|phi>)      <m|a_l|psi>
//     rho2[(k,s),(q,l)] = sum_{m in N-2}  conj(<m|a_k a_s|phi>)  <m|a_q a_l|psi>
// with phi = psi for rho1/rho2 and phi != psi for the transition densities
// <phi|a+_k a_l|psi>, <phi|a+_k a+_s a_q a_l|psi> (for phi != psi every entry
// is reduced; for one state only the Hermitian half of the Gram matrix is
// reduced and the rest is its conjugate transpose). One pass
// over the hole space: a CTA gathers a tile of 32 hole configurations x K
// columns (K = M or P = M(M+1)/2) of <m|A|.> into shared memory, then each
// thread accumulates a 4x4 block of the K x K Gram matrix in registers across
// all tiles of its grid-stride loop. Per-CTA partials go to global memory and
// a second kernel sums them in a fixed order and scatters them into the
// reference layout, so the result is deterministic run to run.
#include <cuda_runtime.h>
#include "fock.cuh"
#include "kernels.h"

namespace mcpi {

namespace {

constexpr int kTile = 32;       // hole configurations per tile
constexpr int kThreads = 256;
constexpr int kGramBlocks = 296;  // 2 x 148 SMs

__device__ __forceinline__ void cfma_conj(double2 &acc, double2 a, double2 b)
{
    // acc += conj(a) * b
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}

template <int M, int ORDER>
struct Cols {
    static constexpr int K = ORDER == 2 ? M * (M + 1) / 2 : M;
    static constexpr int NB = (K + 3) / 4;
    static constexpr int KP = NB * 4;           // padded rows
    static constexpr int LD = kTile + 1;        // row stride (double2), 16 B mod 128 B
};

// Gathers <m|A_c|x> for the tile's hole configurations into D[c*LD + mt].
template <int M, int ORDER>
__device__ __forceinline__ void gather_tile(const Space &sp, const uint32_t *W, const double *sq,
                                           const uint64_t *occ2, int occ_bits, uint32_t m0,
                                           const double2 *__restrict__ x, double2 *D)
{
    using C = Cols<M, ORDER>;
    const int mt = threadIdx.x % kTile, cg = threadIdx.x / kTile;
    constexpr int G = kThreads / kTile;   // column groups
    const uint32_t m = m0 + mt;
    const uint32_t nh = ORDER == 2 ? sp.nc2 : sp.nc1;
    const int ws = sp.wstride;
    if (m >= nh) {
        for (int c = cg; c < C::K; c += G) D[c * C::LD + mt] = make_double2(0.0, 0.0);
        return;
    }
    int u[M], Q[M];
    // decoded here: in this kernel a global load of the packed table per thread
    // measured slower than the shared-memory decode
    (void)occ2;
    (void)occ_bits;
    decode<M>(m, sp.N - ORDER, nh, W, ws, u, Q);
    uint32_t B0[M], B1[M];
    prefix_table<M>(Q, 0, W, ws, B0);
    prefix_table<M>(Q, 1, W, ws, B1);
    if (ORDER == 1) {
#pragma unroll
        for (int l = 0; l < M; ++l) {
            if (l % G != cg) continue;
            const uint32_t j = idx_add1(sp.nc, B0, B1, l, M);
            const double c = sq[u[l] + 1];
            double2 a = x[j];
            D[l * C::LD + mt] = make_double2(c * a.x, c * a.y);
        }
    } else {
        uint32_t B2[M];
        prefix_table<M>(Q, 2, W, ws, B2);
#pragma unroll
        for (int q = 0; q < M; ++q)
#pragma unroll
            for (int l = q; l < M; ++l) {
                const int col = pair_index(q, l, M);
                if (col % G != cg) continue;
                const uint32_t j = idx_add2(sp.nc, B0, B1, B2, q, l, M);
                const double c = (q == l) ? sq[u[q] + 1] * sq[u[q] + 2] : sq[u[q] + 1] * sq[u[l] + 1];
                double2 a = x[j];
                D[col * C::LD + mt] = make_double2(c * a.x, c * a.y);
            }
    }
}

// G partial of this CTA: sum over its tiles of conj(D_phi)^T D_psi, one 4x4
// output block per thread (blockIdx.y selects the group of output blocks).
template <int M, int ORDER, bool SAME>
__global__ void __launch_bounds__(kThreads) k_gram(Space sp, SpaceTables tb,
                                                   const double2 *__restrict__ phi,
                                                   const double2 *__restrict__ psi,
                                                   double2 *__restrict__ partial)
{
    using C = Cols<M, ORDER>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *Dphi = reinterpret_cast<double2 *>(smem_raw);                 // KP x LD
    double2 *Dpsi = SAME ? Dphi : Dphi + C::KP * C::LD;                    // KP x LD
    double *sq = reinterpret_cast<double *>(Dphi + (SAME ? 1 : 2) * C::KP * C::LD);
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);
    for (int x = threadIdx.x; x < (M - 1) * sp.wstride; x += blockDim.x) W[x] = tb.W[x];
    for (int x = threadIdx.x; x < sp.wstride; x += blockDim.x) sq[x] = tb.sq[x];
    // zero the padding rows once
    for (int x = threadIdx.x; x < (C::KP - C::K) * C::LD; x += blockDim.x) {
        Dphi[C::K * C::LD + x] = make_double2(0.0, 0.0);
        if (!SAME) Dpsi[C::K * C::LD + x] = make_double2(0.0, 0.0);
    }

    // output block of this thread: rows aa + r*NB and columns bb + c*NB
    // (r, c < 4). Interleaved rather than four consecutive rows: the row
    // stride LD = 33 double2 puts row x in 16-byte bank slot (x + t) mod 8, so
    // a warp's ~14 distinct bb land on all eight slots (2 wavefronts per load)
    // where the consecutive form (rows 4*bb + c) hit only two (7 wavefronts).
    // With phi = psi the Gram matrix is Hermitian: only the blocks with
    // aa <= bb are reduced (NB(NB+1)/2 of NB^2) and k_gram_finish takes the
    // others as conjugates of their mirror entries.
    const int blk = blockIdx.y * kThreads + threadIdx.x;
    const bool active = blk < (SAME ? C::NB * (C::NB + 1) / 2 : C::NB * C::NB);
    int aa = 0, bb = 0;
    if (active) {
        if (SAME) {
            int rem = blk;
            while (rem >= C::NB - aa) {
                rem -= C::NB - aa;
                ++aa;
            }
            bb = aa + rem;
        } else {
            aa = blk / C::NB;
            bb = blk % C::NB;
        }
    }
    double2 acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = make_double2(0.0, 0.0);

    const uint32_t nh = ORDER == 2 ? sp.nc2 : sp.nc1;
    const uint32_t ntiles = (nh + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        gather_tile<M, ORDER>(sp, W, sq, tb.occ2, tb.occ_bits, tile * kTile, phi, Dphi);
        if (!SAME) gather_tile<M, ORDER>(sp, W, sq, tb.occ2, tb.occ_bits, tile * kTile, psi, Dpsi);
        __syncthreads();
        if (active) {
#pragma unroll 4
            for (int t = 0; t < kTile; ++t) {
                double2 pa[4], pb[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) pa[r] = Dphi[(aa + r * C::NB) * C::LD + t];
#pragma unroll
                for (int c = 0; c < 4; ++c) pb[c] = Dpsi[(bb + c * C::NB) * C::LD + t];
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                    for (int c = 0; c < 4; ++c) cfma_conj(acc[r][c], pa[r], pb[c]);
            }
        }
    }
    if (active) {
        double2 *out = partial + (size_t)blockIdx.x * C::K * C::K;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (aa + r * C::NB < C::K && bb + c * C::NB < C::K)
                    out[(aa + r * C::NB) * C::K + (bb + c * C::NB)] = acc[r][c];
    }
}

// rho1 (and the transition rho1): G[a][b] = sum_h conj(Dphi[a][h]) Dpsi[b][h] over
// the N-1 space with D[l][h] = sqrt(u_l+1) x[index(h + e_l)]. Only M columns, so
// the Gram kernel above would keep one 4x4 block per thread busy (9 threads of
// 256 at M = 10). Here a tile is kTile1 hole configurations, one per thread
// (one decode each); the product gives every thread one entry (a, b) (a <= b
// when phi = psi) and one of S interleaved subsets of the tile's
// configurations; the subsets are summed in a fixed order at the end, so the
// per-CTA partials (same layout as k_gram's) are deterministic.
constexpr int kTile1 = 256;

template <int M, bool SAME>
__global__ void __launch_bounds__(kThreads) k_rho1(Space sp, SpaceTables tb, const double2 *__restrict__ phi,
                                                   const double2 *__restrict__ psi,
                                                   double2 *__restrict__ partial)
{
    constexpr int LD = kTile1 + 1;                              // row stride (double2)
    constexpr int NE = SAME ? M * (M + 1) / 2 : M * M;          // entries
    constexpr int S = NE >= kThreads ? 1 : kThreads / NE;       // configuration subsets
    static_assert(NE <= kThreads, "one entry per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *Dphi = reinterpret_cast<double2 *>(smem_raw);     // M x LD
    double2 *Dpsi = SAME ? Dphi : Dphi + M * LD;
    double2 *red = Dphi + (SAME ? 1 : 2) * M * LD;              // kThreads
    double *sq = reinterpret_cast<double *>(red + kThreads);
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);
    for (int x = threadIdx.x; x < (M - 1) * sp.wstride; x += blockDim.x) W[x] = tb.W[x];
    for (int x = threadIdx.x; x < sp.wstride; x += blockDim.x) sq[x] = tb.sq[x];

    // this thread's entry and subset
    const int t = threadIdx.x;
    const bool active = t < NE * S;
    const int e = active ? t / S : 0, sub = active ? t % S : 0;
    int a = 0, b = 0;
    if (SAME) {
        int rem = e;   // (a, b), a <= b, in pair order
        while (rem >= M - a) {
            rem -= M - a;
            ++a;
        }
        b = a + rem;
    } else {
        a = e / M;
        b = e % M;
    }
    double2 acc = make_double2(0.0, 0.0);

    const uint32_t nh = sp.nc1;
    const uint32_t ntiles = (nh + kTile1 - 1) / kTile1;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        const uint32_t h = tile * kTile1 + t;
        if (h < nh) {
            int u[M], Q[M];
            decode<M>(h, sp.N - 1, nh, W, sp.wstride, u, Q);
            uint32_t B0[M], B1[M];
            prefix_table<M>(Q, 0, W, sp.wstride, B0);
            prefix_table<M>(Q, 1, W, sp.wstride, B1);
#pragma unroll
            for (int l = 0; l < M; ++l) {
                const uint32_t j = idx_add1(sp.nc, B0, B1, l, M);
                const double c = sq[u[l] + 1];
                const double2 x = phi[j];
                Dphi[l * LD + t] = make_double2(c * x.x, c * x.y);
                if (!SAME) {
                    const double2 y = psi[j];
                    Dpsi[l * LD + t] = make_double2(c * y.x, c * y.y);
                }
            }
        } else {
#pragma unroll
            for (int l = 0; l < M; ++l) {
                Dphi[l * LD + t] = make_double2(0.0, 0.0);
                if (!SAME) Dpsi[l * LD + t] = make_double2(0.0, 0.0);
            }
        }
        __syncthreads();
        if (active) {
#pragma unroll 4
            for (int i = sub; i < kTile1; i += S) cfma_conj(acc, Dphi[a * LD + i], Dpsi[b * LD + i]);
        }
    }
    __syncthreads();
    red[t] = acc;
    __syncthreads();
    if (active && sub == 0) {
        double2 g = make_double2(0.0, 0.0);
        for (int k = 0; k < S; ++k) {
            g.x += red[e * S + k].x;
            g.y += red[e * S + k].y;
        }
        double2 *out = partial + (size_t)blockIdx.x * M * M;
        out[a * M + b] = g;
        if (SAME && a != b) out[b * M + a] = make_double2(g.x, -g.y);
    }
}

// Sums the per-CTA partials in block order and writes the reference layout.
// HERM: the partials hold only the blocks of k_gram<.., SAME = true> (entry
// (a, b) with a mod NB <= b mod NB); the rest is conj of the entry (b, a).
template <int M, int ORDER, bool HERM = false>
__global__ void k_gram_finish(const double2 *__restrict__ partial, int nblocks,
                              double2 *__restrict__ out)
{
    using C = Cols<M, ORDER>;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    int a, b;
    if (ORDER == 1) {
        if (x >= M * M) return;
        a = x / M;              // rho1[k*M + l] = G[k][l]
        b = x % M;
    } else {
        if (x >= M * M * M * M) return;
        const int k = x % M, s = (x / M) % M, q = (x / (M * M)) % M, l = x / (M * M * M);
        a = k <= s ? pair_index(k, s, M) : pair_index(s, k, M);
        b = q <= l ? pair_index(q, l, M) : pair_index(l, q, M);
    }
    const bool mirror = HERM && (a % C::NB) > (b % C::NB);
    const int e = mirror ? b * C::K + a : a * C::K + b;
    double2 acc = make_double2(0.0, 0.0);
    for (int blk = 0; blk < nblocks; ++blk) {
        const double2 p = partial[(size_t)blk * C::K * C::K + e];
        acc.x += p.x;
        acc.y += p.y;
    }
    if (mirror) acc.y = -acc.y;
    out[x] = acc;
}

template <int M, int ORDER>
cudaError_t density_m(const Space &sp, const SpaceTables &tb, const double2 *phi,
                      const double2 *psi, double2 *partial, double2 *out, cudaStream_t st)
{
    using C = Cols<M, ORDER>;
    const bool same = (phi == psi);
    if constexpr (ORDER == 1) {
        const size_t smem = sizeof(double2) * ((same ? 1 : 2) * (size_t)M * (kTile1 + 1) + kThreads) +
                            sizeof(double) * sp.wstride + sizeof(uint32_t) * (M - 1) * sp.wstride;
        const unsigned ntiles = (sp.nc1 + kTile1 - 1) / kTile1;
        const unsigned gx = ntiles < (unsigned)kGramBlocks ? (ntiles ? ntiles : 1) : kGramBlocks;
        cudaError_t e;
        if (same) {
            e = cudaFuncSetAttribute(k_rho1<M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            k_rho1<M, true><<<gx, kThreads, smem, st>>>(sp, tb, phi, psi, partial);
        } else {
            e = cudaFuncSetAttribute(k_rho1<M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            k_rho1<M, false><<<gx, kThreads, smem, st>>>(sp, tb, phi, psi, partial);
        }
        k_gram_finish<M, 1><<<(M * M + 255) / 256, 256, 0, st>>>(partial, gx, out);
        return cudaGetLastError();
    }
    const size_t tiles = sizeof(double2) * C::KP * C::LD * (same ? 1 : 2);
    const size_t smem = tiles + sizeof(double) * sp.wstride + sizeof(uint32_t) * (M - 1) * sp.wstride;
    const uint32_t nh = ORDER == 2 ? sp.nc2 : sp.nc1;
    const unsigned ntiles = (nh + kTile - 1) / kTile;
    const unsigned gx = ntiles < (unsigned)kGramBlocks ? (ntiles ? ntiles : 1) : kGramBlocks;
    const unsigned nblk = same ? C::NB * (C::NB + 1) / 2 : C::NB * C::NB;
    const unsigned gy = (nblk + kThreads - 1) / kThreads;
    dim3 grid(gx, gy);
    cudaError_t e;
    if (same) {
        e = cudaFuncSetAttribute(k_gram<M, ORDER, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_gram<M, ORDER, true><<<grid, kThreads, smem, st>>>(sp, tb, phi, psi, partial);
    } else {
        e = cudaFuncSetAttribute(k_gram<M, ORDER, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_gram<M, ORDER, false><<<grid, kThreads, smem, st>>>(sp, tb, phi, psi, partial);
    }
    const int nout = ORDER == 1 ? M * M : M * M * M * M;
    if (same)
        k_gram_finish<M, ORDER, true><<<(nout + 255) / 256, 256, 0, st>>>(partial, gx, out);
    else
        k_gram_finish<M, ORDER, false><<<(nout + 255) / 256, 256, 0, st>>>(partial, gx, out);
    return cudaGetLastError();
}

}  // namespace

size_t gram_partial_elems(const Space &sp, int order)
{
    const int K = order == 2 ? sp.M * (sp.M + 1) / 2 : sp.M;
    return (size_t)kGramBlocks * K * K;
}

cudaError_t launch_density(const Space &sp, const SpaceTables &tb, int order, const double2 *phi,
                           const double2 *psi, double2 *partial, double2 *out, cudaStream_t st)
{
    const int nout = order == 1 ? sp.M * sp.M : sp.M * sp.M * sp.M * sp.M;
    if (sp.N < order) return cudaMemsetAsync(out, 0, sizeof(double2) * nout, st);
    switch (sp.M * 4 + order) {
#define MCPI_CASE(m)                                                                      \
    case m * 4 + 1: return density_m<m, 1>(sp, tb, phi, psi, partial, out, st);          \
    case m * 4 + 2: return density_m<m, 2>(sp, tb, phi, psi, partial, out, st);
        MCPI_CASE(1) MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6)
        MCPI_CASE(7) MCPI_CASE(8) MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12)
        MCPI_CASE(13) MCPI_CASE(14) MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace mcpi
