// Fock-space arithmetic shared by every kernel and by the host planner.
//
// Ordering. The reference's perfect hash (configurationsMap.h:273-305,
// FockToIndex) empties orbitals from the top, each particle of orbital i
// adding NC(n_remaining, i), NC(n,m) = C(n+m-1, n). Summing that series with
// the hockey-stick identity gives a closed form in the prefix counts
// P_i = v_0 + ... + v_i of an n-particle configuration v:
//
//     index(v) = NC(n,M) - 1 - sum_{i=0}^{M-2} W_i(P_i),   W_i(p) = C(p+i, i+1).
//
// The formula depends on n only through NC(n,M), so one table W serves the N,
// N-1 and N-2 particle spaces alike. A jump that removes or adds particles
// shifts the prefix counts by a step function of the orbital (e.g. removing
// e_k + e_s, k <= s, lowers P_i by 1 on [k,s) and by 2 on [s,M-1]), so with
// per-configuration prefix sums  A_d[t] = sum_{i<t} W_i(P_i + d)  the index of
// any one- or two-particle jump is a difference of a few table entries: O(1)
// per jump instead of the reference's O(M) hash or its stored maps.
//
// Decoding an index back to occupations (configurationsMap.h:238-269,
// IndexToFock) is the greedy inverse: R = NC(n,M)-1-index is a sum of
// binomials with strictly increasing upper arguments (a combinatorial number
// system), so P_{M-2}, P_{M-3}, ... are found from the top by decreasing p
// while W_i(p) > R.
//
// Index arithmetic is 32-bit unsigned. The host rejects spaces with
// NC(N,M) >= 2^31; every W entry a valid jump needs is then < 2^31, and
// out-of-range entries that cancel in a difference wrap modulo 2^32 harmlessly.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define MCPI_HD __host__ __device__ __forceinline__
#else
#define MCPI_HD inline
#endif

namespace mcpi {

constexpr int kMaxM = 16;                      // orbitals supported by the kernels
constexpr int kMaxPairs = kMaxM * (kMaxM + 1) / 2;

// Pair (k <= s) -> column. Row-major upper triangle: (0,0),(0,1)..(0,M-1),(1,1)..
MCPI_HD int pair_index(int k, int s, int M) { return k * M - (k * (k - 1)) / 2 + (s - k); }

// Geometry of one Fock space, passed by value to kernels.
struct Space {
    int N, M;          // particles, orbitals
    int wstride;       // row stride of the W table (= N + 3)
    int pad;
    uint32_t nc;       // NC(N,M)
    uint32_t nc1;      // NC(N-1,M)  (0 when N < 1)
    uint32_t nc2;      // NC(N-2,M)  (0 when N < 2)
    uint32_t pad2;
};

// W_i(p) lookup with p clamped at 0 from below (negative p only occurs in
// entries that cancel).
MCPI_HD uint32_t wlook(const uint32_t *W, int ws, int i, int p) { return p < 0 ? 0u : W[i * ws + p]; }

// Decode index -> occupations v[0..M-1] and prefix counts P[0..M-1] of an
// n-particle configuration (ncn = NC(n,M)).
template <int M>
MCPI_HD void decode(uint32_t idx, int n, uint32_t ncn, const uint32_t *W, int ws, int *v, int *P)
{
    uint32_t R = ncn - 1u - idx;
    int hi = n;
    P[M - 1] = n;
#pragma unroll
    for (int i = M - 2; i >= 0; --i) {
        int p = hi;
        while (p > 0 && W[i * ws + p] > R) --p;
        R -= W[i * ws + p];
        P[i] = p;
        hi = p;
    }
    v[0] = P[0];
#pragma unroll
    for (int i = 1; i < M; ++i) v[i] = P[i] - P[i - 1];
}

// Occupations v and prefix counts P of configuration idx of an n-particle
// space: from the packed table when there is one, else by decoding the index.
template <int M>
MCPI_HD void occupations(const uint64_t *occ, int bits, uint32_t idx, int n, uint32_t ncn,
                                            const uint32_t *W, int ws, int *v, int *P)
{
    if (occ) {
        const uint64_t w = occ[idx];
        const uint32_t mask = (1u << bits) - 1u;
        int run = 0;
#pragma unroll
        for (int q = 0; q < M; ++q) {
            v[q] = (int)((w >> (bits * q)) & mask);
            run += v[q];
            P[q] = run;
        }
    } else {
        decode<M>(idx, n, ncn, W, ws, v, P);
    }
}

// Prefix sums A[t] = sum_{i<t} W_i(P_i + d), t = 0..M-1 (A[M-1] is the full sum).
template <int M>
MCPI_HD void prefix_table(const int *P, int d, const uint32_t *W, int ws, uint32_t *A)
{
    uint32_t acc = 0;
    A[0] = 0;
#pragma unroll
    for (int t = 1; t < M; ++t) {
        acc += wlook(W, ws, t - 1, P[t - 1] + d);
        A[t] = acc;
    }
}

// Index in the (n-2)-space of v - e_k - e_s (k <= s), from the tables of v
// with d = 0, -1, -2 (A0, Am1, Am2). ncm2 = NC(n-2,M).
MCPI_HD uint32_t idx_remove2(uint32_t ncm2, const uint32_t *A0, const uint32_t *Am1,
                             const uint32_t *Am2, int k, int s, int M)
{
    return ncm2 - 1u - (A0[k] + (Am1[s] - Am1[k]) + (Am2[M - 1] - Am2[s]));
}

// Index in the (n+2)-space of u + e_q + e_l (q <= l), from the tables of u
// with d = 0, +1, +2. ncp2 = NC(n+2,M).
MCPI_HD uint32_t idx_add2(uint32_t ncp2, const uint32_t *B0, const uint32_t *B1,
                          const uint32_t *B2, int q, int l, int M)
{
    return ncp2 - 1u - (B0[q] + (B1[l] - B1[q]) + (B2[M - 1] - B2[l]));
}

// Index in the (n+1)-space of u + e_l, from the tables of u with d = 0, +1.
MCPI_HD uint32_t idx_add1(uint32_t ncp1, const uint32_t *B0, const uint32_t *B1, int l, int M)
{
    return ncp1 - 1u - (B0[l] + (B1[M - 1] - B1[l]));
}

// Index in the (n-1)-space of v - e_k, from the tables of v with d = 0, -1.
MCPI_HD uint32_t idx_remove1(uint32_t ncm1, const uint32_t *A0, const uint32_t *Am1, int k, int M)
{
    return ncm1 - 1u - (A0[k] + (Am1[M - 1] - Am1[k]));
}

// Index in the same space of v - e_k + e_l (one particle moved k -> l), from
// the tables of v with d = 0, -1, +1.
MCPI_HD uint32_t idx_move1(uint32_t ncn, const uint32_t *A0, const uint32_t *Am1,
                           const uint32_t *Ap1, int k, int l, int M)
{
    // P shifts by -1 on [k,l) when k < l, by +1 on [l,k) when l < k.
    if (k == l) return ncn - 1u - A0[M - 1];
    if (k < l) return ncn - 1u - (A0[M - 1] - (A0[l] - A0[k]) + (Am1[l] - Am1[k]));
    return ncn - 1u - (A0[M - 1] - (A0[k] - A0[l]) + (Ap1[k] - Ap1[l]));
}

}  // namespace mcpi
