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
constexpr int kT2 = 256;   // threads per block, kernel 2

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
    double *sq = reinterpret_cast<double *>(D + P * kT1);           // wstride
    uint32_t *W = reinterpret_cast<uint32_t *>(sq + sp.wstride);    // (M-1) x wstride
    load_tables(sp, tb, W, sq);
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
        const int z0 = __ldg(op.rowptr + a), z1 = __ldg(op.rowptr + a + 1);
        double2 e = make_double2(0.0, 0.0);
        for (int z = z0; z < z1; ++z) {
            const double2 h = __ldg(op.val + z);
            const int b = __ldg(op.col + z);
            cfma(e, h, Dt[b * kT1]);
        }
        E[a * stride + m] = e;
    }
}

// ---------------------------------------------------------------------------
// kernel 2: out[i] = (sum_k Ho[k][k] v_k) psi[i] + sum_a c_a(v) E[a][index(v - pair a)]
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kT2) k_pair_create(Space sp, SpaceTables tb, PairOp op,
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
        uint32_t A0[M], Am1[M], Am2[M];
        prefix_table<M>(P, 0, W, ws, A0);
        prefix_table<M>(P, -1, W, ws, Am1);
        prefix_table<M>(P, -2, W, ws, Am2);
        const size_t stride = sp.nc2;
#pragma unroll
        for (int k = 0; k < M; ++k)
#pragma unroll
            for (int s = k; s < M; ++s) {
                const bool ok = (s == k) ? (v[k] >= 2) : (v[k] >= 1 && v[s] >= 1);
                if (ok) {
                    const uint32_t mm = idx_remove2(sp.nc2, A0, Am1, Am2, k, s, M);
                    const double c = (s == k) ? sq[v[k]] * sq[v[k] - 1] : sq[v[k]] * sq[v[s]];
                    const double2 e = E[pair_index(k, s, M) * stride + mm];
                    acc.x = fma(c, e.x, acc.x);
                    acc.y = fma(c, e.y, acc.y);
                }
            }
    }
    out[i] = acc;
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
cudaError_t apply_h_m(const Space &sp, const SpaceTables &tb, const PairOp &op,
                      const double2 *psi, double2 *E, double2 *out, cudaStream_t st)
{
    constexpr int P = M * (M + 1) / 2;
    const size_t tab = sizeof(double) * sp.wstride + sizeof(uint32_t) * (M - 1) * sp.wstride;
    if (sp.N >= 2) {
        const size_t sm1 = sizeof(double2) * P * kT1 + tab;
        if (sm1 > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(
                k_pair_annihilate<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
            if (e != cudaSuccess) return e;
        }
        const unsigned g1 = (sp.nc2 + kT1 - 1) / kT1;
        k_pair_annihilate<M><<<g1, kT1, sm1, st>>>(sp, tb, op, psi, E);
    }
    const size_t sm2 = sizeof(double2) * M + tab;
    const unsigned g2 = (sp.nc + kT2 - 1) / kT2;
    k_pair_create<M><<<g2, kT2, sm2, st>>>(sp, tb, op, psi, E, out);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_apply_h(const Space &sp, const SpaceTables &tb, const PairOp &op,
                           const double2 *psi, double2 *E, double2 *out, cudaStream_t st)
{
    if (sp.N == 1) {
        k_one_particle<<<1, 32, 0, st>>>(sp.M, op.hfull, psi, out);
        return cudaGetLastError();
    }
    switch (sp.M) {
#define MCPI_CASE(m) \
    case m: return apply_h_m<m>(sp, tb, op, psi, E, out, st);
        MCPI_CASE(1) MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6)
        MCPI_CASE(7) MCPI_CASE(8) MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12)
        MCPI_CASE(13) MCPI_CASE(14) MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace mcpi
