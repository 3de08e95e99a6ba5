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
#include "mbarrier.cuh"

namespace mcpi {

namespace {

constexpr int kTile = 32;       // hole configurations per tile
constexpr int kThreads = 256;
constexpr int kGramBlocks = 296;  // 2 x 148 SMs
constexpr int kDmmaBlocks = 148;  // one persistent block per SM (fixed: it sets the reduction order)

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

// ---------------------------------------------------------------------------
// rho2 and the transition rho2 on the FP64 tensor cores (M <= 12).
// G[a][b] = sum_m conj(Dphi[a][m]) Dpsi[b][m] is a K x K product reduced over
// the (N-2) space, K = M(M+1)/2: with mma.sync.m16n8k4.f64 the rows are pairs
// a (16 per MMA), the columns pairs b (8 per MMA) and the reduction runs over
// configurations m (4 per MMA). The complex product takes three real ones
// (Gauss): t1 += Ar Br, t2 += Ai Bi, t3 += (Ar - Ai)(Br + Bi), and at the end
// Re G = t1 + t2, Im G = t3 - t1 + t2 (A = Dphi, conjugated by the signs).
// One persistent block per SM, warp-specialised: gather warps fill tiles of
// GM configurations (one decode per configuration, K scattered 16-byte loads
// of each vector from L2, the factors c_b(m), real and imaginary parts into
// separate row-major planes) into two stages; 8 product warps each own a
// fixed set of 16 x 8 output tiles and keep their accumulators in registers
// across all of the block's configuration tiles. With one state the Gram
// matrix is Hermitian: only the tiles (i, j) with j >= 2i are reduced (16 of
// 28 at M = 10) and the finish kernel takes the others as conjugates of their
// mirror entries. Hand-over by mbarriers whose waits are bounded (about two
// seconds; then the status word reports MCPI_ERR_TIMEOUT). Per-block partials
// are summed in block order by k_gram_finish: deterministic.
// Plane layout: row r (pair) at r * LD doubles, LD = GM + 4, so the 8 rows x 4
// consecutive configurations of one fragment load fall into distinct banks.
// ---------------------------------------------------------------------------
constexpr int kDmmaPW = 8;                            // product warps
constexpr int kDmmaStages = 2;
constexpr int kDmmaUnroll = 4;   // configuration steps of the product loop unrolled together
constexpr int kDmmaMaxM = 12;        // rho2 of one state
constexpr int kDmmaMaxMTrans = 10;   // transition rho2 (more accumulators: larger M would spill)

template <int M, bool SAME>
struct DmmaGram {
    static constexpr int K = M * (M + 1) / 2;
    static constexpr int AG = (K + 15) / 16;         // 16-row groups of a
    static constexpr int BG = (K + 7) / 8;           // 8-column groups of b
    static constexpr int KP = AG * 16;               // padded plane rows (>= BG * 8)
    // SUMS: the gather warps form the Gauss sum planes Ar - Ai and Br + Bi
    // (the transition form: measured 4.45 against 4.70 ms at N=20, M=10);
    // otherwise the product warps add the fragments themselves (one state:
    // half the planes, so tiles of 64 configurations fit two stages -- with
    // sum planes and 32-configuration tiles it took 4.6 against 2.9 ms).
    static constexpr bool SUMS = !SAME;
    // ASUM (one state, M <= 10): the gather warps also write the A-side sum
    // plane Ar - Ai, so the product warps' FP64 adds -- on the pipe the DMMAs
    // use -- are only the B-side sums; three planes of 64 configurations fit
    // two stages in shared memory up to 64 padded rows
    static constexpr bool ASUM = SAME && KP <= 64;
    static constexpr int NP = SAME ? (ASUM ? 3 : 2) : 6;
    static constexpr int GM = SAME ? 64 : 32;        // configurations per tile
    static constexpr int LD = GM + 4;                // plane row stride (doubles)
    // gather warps: 8 for one state up to M = 10 (four threads per
    // configuration of a 64-configuration tile), else 4 (the transition form
    // loads two vectors, and M > 10 has more accumulators: with 8 warps, 128
    // registers per thread would spill)
    static constexpr int GW = (SAME && M <= 10) ? 8 : 4;
    static constexpr int THREADS = (kDmmaPW + GW) * 32;
    static constexpr int GT = GW * 32;               // gather threads
    static constexpr int PARTS = GT / GM;            // gather threads per configuration
    static constexpr int ntiles()
    {
        int n = 0;
        for (int i = 0; i < AG; ++i)
            for (int j = 0; j < BG; ++j)
                if (!SAME || j >= 2 * i) ++n;
        return n;
    }
    static constexpr int NT = ntiles();
    static constexpr int TPW = (NT + kDmmaPW - 1) / kDmmaPW;   // most tiles of one product warp
    // product warp w takes tiles [tstart(w), tstart(w) + tcount(w)): the tiles
    // split as evenly as they go, so warps w and w + 4, which share an SM
    // sub-partition's tensor core, hold nearly the same work (the transition
    // form at M = 10: 28 tiles as 4,4,4,4,3,3,3,3 rather than seven warps of 4)
    static constexpr __host__ __device__ int tcount(int w) { return NT / kDmmaPW + (w < NT % kDmmaPW ? 1 : 0); }
    static constexpr __host__ __device__ int tstart(int w)
    {
        return w * (NT / kDmmaPW) + (w < NT % kDmmaPW ? w : NT % kDmmaPW);
    }
    static constexpr size_t stage_bytes = sizeof(double) * NP * KP * LD;
    // planes, then the stage barriers, then the space's sqrt and binomial tables
    static size_t smem(int ws)
    {
        return kDmmaStages * stage_bytes + 2 * kDmmaStages * sizeof(uint64_t) + sizeof(double) * ws +
               sizeof(uint32_t) * (M - 1) * ws;
    }
};

// Output tile n (in i-major order over the kept tiles) -> (i, j).
template <int M, bool SAME>
__device__ __forceinline__ void dmma_tile(int n, int &i, int &j)
{
    using D = DmmaGram<M, SAME>;
    i = 0;
    j = 0;
    for (int a = 0; a < D::AG; ++a) {
        const int j0 = SAME ? 2 * a : 0;
        const int cnt = D::BG > j0 ? D::BG - j0 : 0;
        if (n < cnt) {
            i = a;
            j = j0 + n;
            return;
        }
        n -= cnt;
    }
}

__device__ __forceinline__ void dmma_m16n8k4(double (&c)[4], double a0, double a1, double b)
{
    asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, {%0, %1, %2, %3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b));
}

// One gather thread's share of a tile: configuration m (tile column ml), the
// pair columns col with col % PARTS == PART. All of its loads are issued
// before any is consumed (the columns are compile-time constants, so the
// loaded values stay in registers), then the scaled values and the Gauss sum
// planes go to the stage's planes pl.
template <int M, bool SAME, int PART>
__device__ __forceinline__ void dmma_gather(const Space &sp, const SpaceTables &tb, const uint32_t *W,
                                            const double *sq, const double2 *__restrict__ phi,
                                            const double2 *__restrict__ psi, double *pl, uint32_t m, int ml)
{
    using D = DmmaGram<M, SAME>;
    constexpr int K = D::K, KP = D::KP, LD = D::LD, PARTS = D::PARTS;
    constexpr int NPP = (K + PARTS - 1 - PART) / PARTS;   // my columns
    if (m >= sp.nc2) {
#pragma unroll
        for (int k = 0; k < NPP; ++k)
#pragma unroll
            for (int p = 0; p < D::NP; ++p) pl[(p * KP + PART + k * PARTS) * LD + ml] = 0.0;
        return;
    }
    const int ws = sp.wstride;
    int u[M], Q[M];
    occupations<M>(tb.occ2, tb.occ_bits, m, sp.N - 2, sp.nc2, W, ws, u, Q);
    uint32_t B0[M], B1[M], B2[M];
    prefix_table<M>(Q, 0, W, ws, B0);
    prefix_table<M>(Q, 1, W, ws, B1);
    prefix_table<M>(Q, 2, W, ws, B2);
    double2 x[NPP > 0 ? NPP : 1], y[SAME ? 1 : (NPP > 0 ? NPP : 1)];
    {
        int k = 0;
#pragma unroll
        for (int q = 0; q < M; ++q)
#pragma unroll
            for (int l = q; l < M; ++l)
                if (pair_index(q, l, M) % PARTS == PART) {
                    const uint32_t j = idx_add2(sp.nc, B0, B1, B2, q, l, M);
                    x[k] = __ldg(phi + j);
                    if constexpr (!SAME) y[k] = __ldg(psi + j);
                    ++k;
                }
    }
    int k = 0;
#pragma unroll
    for (int q = 0; q < M; ++q)
#pragma unroll
        for (int l = q; l < M; ++l)
            if (pair_index(q, l, M) % PARTS == PART) {
                const int col = pair_index(q, l, M);
                const double c = (q == l) ? sq[u[q] + 1] * sq[u[q] + 2] : sq[u[q] + 1] * sq[u[l] + 1];
                const double xr = c * x[k].x, xi = c * x[k].y;
                pl[col * LD + ml] = xr;
                pl[(KP + col) * LD + ml] = xi;
                if constexpr (D::ASUM) pl[(2 * KP + col) * LD + ml] = xr - xi;
                if constexpr (D::SUMS) {
                    const double yr = c * y[k].x, yi = c * y[k].y;
                    pl[(2 * KP + col) * LD + ml] = xr - xi;
                    pl[(3 * KP + col) * LD + ml] = yr;
                    pl[(4 * KP + col) * LD + ml] = yi;
                    pl[(5 * KP + col) * LD + ml] = yr + yi;
                }
                ++k;
            }
}

template <int M, bool SAME>
__global__ void __launch_bounds__(DmmaGram<M, SAME>::THREADS, 1)
    k_gram_dmma(Space sp, SpaceTables tb, const double2 *__restrict__ phi, const double2 *__restrict__ psi,
                double2 *__restrict__ partial, int *status, long long wait_cycles, int test_stall)
{
    using D = DmmaGram<M, SAME>;
    constexpr int K = D::K, KP = D::KP, LD = D::LD, GM = D::GM;
    const long long limit = wait_cycles > 0 ? wait_cycles : kWaitCycles;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *planes = reinterpret_cast<double *>(smem_raw);                    // stages x NP x KP x LD
    uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw + kDmmaStages * D::stage_bytes);
    uint64_t *empty = full + kDmmaStages;
    double *sq = reinterpret_cast<double *>(empty + kDmmaStages);          // wstride
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);          // (M-1) x wstride
    const int ws = sp.wstride;
    for (int x = threadIdx.x; x < (M - 1) * ws; x += blockDim.x) W[x] = tb.W[x];
    for (int x = threadIdx.x; x < ws; x += blockDim.x) sq[x] = tb.sq[x];
    // padding rows K .. KP-1 of every plane stay zero
    for (int x = threadIdx.x; x < kDmmaStages * D::NP * (KP - K) * LD; x += blockDim.x) {
        const int per = (KP - K) * LD, pl = x / per, r = x % per;
        planes[(size_t)pl * KP * LD + K * LD + r] = 0.0;
    }
    if (threadIdx.x == 0)
        for (int b = 0; b < kDmmaStages; ++b) {
            mbar_init(full + b, D::GT);
            mbar_init(empty + b, kDmmaPW);
        }
    __syncthreads();

    const uint32_t nh = sp.nc2;
    const uint32_t ntiles = (nh + GM - 1) / GM;
    const uint32_t ntb = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp >= kDmmaPW) {
        // gather: configuration ml of the tile, pair columns col % PARTS == part
        const int g = threadIdx.x - kDmmaPW * 32;
        const int ml = g % GM, part = g / GM;
        for (uint32_t it = 0; it < ntb; ++it) {
            const int st = it % kDmmaStages;
            if (test_stall) return;   // test switch: deliver nothing, so that the product warps' waits run out
            if (it >= kDmmaStages && !mbar_wait(empty + st, (it / kDmmaStages - 1) & 1, limit)) {
                if (status) atomicExch(status, 1);
                return;
            }
            double *pl = planes + (size_t)st * D::NP * KP * LD;
            const uint32_t m = (blockIdx.x + it * gridDim.x) * GM + ml;
            switch (part) {   // the part as a template argument: its pair columns are compile-time constants
            case 0: dmma_gather<M, SAME, 0>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            case 1: dmma_gather<M, SAME, 1>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            case 2: dmma_gather<M, SAME, 2>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            case 3: dmma_gather<M, SAME, 3>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            case 4: if constexpr (D::PARTS > 4) dmma_gather<M, SAME, 4>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            case 5: if constexpr (D::PARTS > 5) dmma_gather<M, SAME, 5>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            case 6: if constexpr (D::PARTS > 6) dmma_gather<M, SAME, 6>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            case 7: if constexpr (D::PARTS > 7) dmma_gather<M, SAME, 7>(sp, tb, W, sq, phi, psi, pl, m, ml); break;
            default: break;
            }
            mbar_arrive(full + st);
        }
        return;
    }

    // product warps: tiles n = tstart(warp) + x, x < tcount(warp)
    const int gq = lane >> 2, tq = lane & 3;
    double acc[D::TPW][3][4];
#pragma unroll
    for (int x = 0; x < D::TPW; ++x)
#pragma unroll
        for (int y = 0; y < 3; ++y)
#pragma unroll
            for (int z = 0; z < 4; ++z) acc[x][y][z] = 0.0;
    int ti[D::TPW], tj[D::TPW];
    const int t0 = D::tstart(warp), tn = D::tcount(warp);
#pragma unroll
    for (int x = 0; x < D::TPW; ++x) dmma_tile<M, SAME>(t0 + (x < tn ? x : 0), ti[x], tj[x]);
    for (uint32_t it = 0; it < ntb; ++it) {
        const int st = it % kDmmaStages;
        if (!mbar_wait(full + st, (it / kDmmaStages) & 1, limit)) {
            if (lane == 0 && status) atomicExch(status, 1);
            return;
        }
        const double *Ar = planes + (size_t)st * D::NP * KP * LD;
        const double *Ai = Ar + KP * LD;
        const double *As = Ar + 2 * KP * LD;                                      // SUMS, ASUM
        const double *Br = SAME ? Ar : Ar + 3 * KP * LD;
        const double *Bi = SAME ? Ai : Ar + 4 * KP * LD;
        const double *Bs = Ar + 5 * KP * LD;                                      // SUMS only
#pragma unroll kDmmaUnroll
        for (int s = 0; s < GM / 4; ++s) {
            const int cm = 4 * s + tq;
            int icur = -1;
            double ar0 = 0, ar1 = 0, ai0 = 0, ai1 = 0, as0 = 0, as1 = 0;
#pragma unroll
            for (int x = 0; x < D::TPW; ++x) {
                if (x >= tn) break;
                if (ti[x] != icur) {   // warp-uniform: reload A only for a new row group
                    icur = ti[x];
                    const int r0 = (16 * icur + gq) * LD + cm, r1 = r0 + 8 * LD;
                    ar0 = Ar[r0];
                    ar1 = Ar[r1];
                    ai0 = Ai[r0];
                    ai1 = Ai[r1];
                    if constexpr (D::SUMS || D::ASUM) {
                        as0 = As[r0];
                        as1 = As[r1];
                    } else {
                        as0 = ar0 - ai0;
                        as1 = ar1 - ai1;
                    }
                }
                const int rb = (8 * tj[x] + gq) * LD + cm;
                const double br = Br[rb], bi = Bi[rb];
                dmma_m16n8k4(acc[x][0], ar0, ar1, br);
                dmma_m16n8k4(acc[x][1], ai0, ai1, bi);
                dmma_m16n8k4(acc[x][2], as0, as1, D::SUMS ? Bs[rb] : br + bi);
            }
        }
        __syncwarp();
        if (lane == 0 && it + kDmmaStages < ntb) mbar_arrive(empty + st);
    }
    double2 *out = partial + (size_t)blockIdx.x * K * K;
#pragma unroll
    for (int x = 0; x < D::TPW; ++x) {
        if (x >= tn) break;
#pragma unroll
        for (int z = 0; z < 4; ++z) {
            const int a = 16 * ti[x] + gq + (z >= 2 ? 8 : 0), b = 8 * tj[x] + 2 * tq + (z & 1);
            if (a < K && b < K) {
                const double t1 = acc[x][0][z], t2 = acc[x][1][z], t3 = acc[x][2][z];
                out[a * K + b] = make_double2(t1 + t2, t3 - t1 + t2);
            }
        }
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
            occupations<M>(tb.occ1, tb.occ_bits, h, sp.N - 1, nh, W, sp.wstride, u, Q);
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
// HERM 1: the partials hold only the blocks of k_gram<.., SAME = true> (entry
// (a, b) with a mod NB <= b mod NB); HERM 2: only the tiles of
// k_gram_dmma<.., SAME = true> (entry (a, b) with b / 8 >= 2 (a / 16)). The
// rest is the conjugate of the entry (b, a), which is then held.
template <int M, int ORDER, int HERM = 0>
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
    const bool mirror = HERM == 1 ? (a % C::NB) > (b % C::NB) : HERM == 2 ? (b / 8) < 2 * (a / 16) : false;
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
                      const double2 *psi, double2 *partial, double2 *out, cudaStream_t st, int *status,
                      long long wait_cycles, int test_stall)
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
    if constexpr (ORDER == 2 && M >= 2 && M <= kDmmaMaxM) {
        // FP64 tensor cores (the transition form up to kDmmaMaxMTrans), when the
        // stages and the space's tables fit the block's shared memory
        const int nout = M * M * M * M;
        int dev = 0, optin = 0;
        cudaError_t qe = cudaGetDevice(&dev);
        if (qe == cudaSuccess) qe = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (qe != cudaSuccess) return qe;
        if (same && DmmaGram<M, true>::smem(sp.wstride) <= (size_t)optin) {
            using Dm = DmmaGram<M, true>;
            const unsigned ntiles = (sp.nc2 + Dm::GM - 1) / Dm::GM;
            const unsigned gx = ntiles < (unsigned)kDmmaBlocks ? (ntiles ? ntiles : 1) : kDmmaBlocks;
            const size_t sm = Dm::smem(sp.wstride);
            cudaError_t e = cudaFuncSetAttribute(k_gram_dmma<M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            if (e != cudaSuccess) return e;
            k_gram_dmma<M, true><<<gx, Dm::THREADS, sm, st>>>(sp, tb, phi, psi, partial, status, wait_cycles,
                                                               test_stall);
            k_gram_finish<M, 2, 2><<<(nout + 255) / 256, 256, 0, st>>>(partial, gx, out);
            return cudaGetLastError();
        }
        if constexpr (M <= kDmmaMaxMTrans) {
            if (!same && DmmaGram<M, false>::smem(sp.wstride) <= (size_t)optin) {
            using Dm = DmmaGram<M, false>;
            const unsigned ntiles = (sp.nc2 + Dm::GM - 1) / Dm::GM;
            const unsigned gx = ntiles < (unsigned)kDmmaBlocks ? (ntiles ? ntiles : 1) : kDmmaBlocks;
            const size_t sm = Dm::smem(sp.wstride);
            cudaError_t e = cudaFuncSetAttribute(k_gram_dmma<M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            if (e != cudaSuccess) return e;
            k_gram_dmma<M, false><<<gx, Dm::THREADS, sm, st>>>(sp, tb, phi, psi, partial, status, wait_cycles,
                                                                test_stall);
            k_gram_finish<M, 2, 0><<<(nout + 255) / 256, 256, 0, st>>>(partial, gx, out);
            return cudaGetLastError();
            }
        }
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
        k_gram_finish<M, ORDER, 1><<<(nout + 255) / 256, 256, 0, st>>>(partial, gx, out);
    else
        k_gram_finish<M, ORDER, 0><<<(nout + 255) / 256, 256, 0, st>>>(partial, gx, out);
    return cudaGetLastError();
}

}  // namespace

size_t gram_partial_elems(const Space &sp, int order)
{
    const int K = order == 2 ? sp.M * (sp.M + 1) / 2 : sp.M;
    return (size_t)kGramBlocks * K * K;
}

cudaError_t launch_density(const Space &sp, const SpaceTables &tb, int order, const double2 *phi,
                           const double2 *psi, double2 *partial, double2 *out, cudaStream_t st, int *status,
                           long long wait_cycles, int test_stall)
{
    const int nout = order == 1 ? sp.M * sp.M : sp.M * sp.M * sp.M * sp.M;
    if (sp.N < order) return cudaMemsetAsync(out, 0, sizeof(double2) * nout, st);
    switch (sp.M * 4 + order) {
#define MCPI_CASE(m)                                                                      \
    case m * 4 + 1: return density_m<m, 1>(sp, tb, phi, psi, partial, out, st, status, wait_cycles, test_stall); \
    case m * 4 + 2: return density_m<m, 2>(sp, tb, phi, psi, partial, out, st, status, wait_cycles, test_stall);
        MCPI_CASE(1) MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6)
        MCPI_CASE(7) MCPI_CASE(8) MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12)
        MCPI_CASE(13) MCPI_CASE(14) MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace mcpi
