// The two-body pair matrix of H, shared by every host path that builds one.
//
// Ht[a][b] (a = (k<=s) creation pair, b = (q<=l) annihilation pair, both in
// pair_index order) is such that  sum_ab Ht[a][b] a+_k a+_s a_q a_l  equals the
// reference's two-body sum rule by rule (hamiltonianMatrix.h:976-1418; each
// rule's factor 1, 2 or 4 times the outer 1/2, on the Hint entry that rule
// reads; variant MCPI_VARIANT_HASH sums Rule 9 over all orderings with weight
// 1 as applyHconf does, hamiltonianMatrix.h:390-416), plus the off-diagonal
// one-body part folded in as a+_k a_l = (N-1)^-1 sum_s a+_k a+_s a_s a_l.
//
// The caller provides Ht (P*P entries, P = M(M+1)/2), so the allocation-free
// entry point can fold into a buffer of its own; every path runs these same
// additions in this same order and gets bitwise the same matrix.
#pragma once
#include <complex>

#include "fock.cuh"

namespace mcpi {

inline void fold_pair_matrix(int N, int M, const std::complex<double> *Ho, const std::complex<double> *Hint,
                             bool hash_variant, std::complex<double> *Ht)
{
    using cplx = std::complex<double>;
    const int P = M * (M + 1) / 2;
    const size_t M2 = (size_t)M * M, M3 = M2 * M;
    for (int x = 0; x < P * P; ++x) Ht[x] = cplx(0.0, 0.0);
    if (N < 2) return;
    auto H = [&](int k, int s, int q, int l) { return Hint[k + s * M + q * M2 + l * M3]; };
    auto pr = [&](int a, int b) { return a <= b ? pair_index(a, b, M) : pair_index(b, a, M); };
    auto at = [&](int a, int b) -> cplx & { return Ht[(size_t)a * P + b]; };
    for (int k = 0; k < M; ++k) at(pr(k, k), pr(k, k)) += 0.5 * H(k, k, k, k);           // R1
    for (int k = 0; k < M; ++k)                                                           // R2
        for (int s = k + 1; s < M; ++s) at(pr(k, s), pr(k, s)) += 2.0 * H(k, s, k, s);
    for (int k = 0; k < M; ++k)                                                           // R3
        for (int q = 0; q < M; ++q)
            if (q != k) at(pr(k, k), pr(q, q)) += 0.5 * H(k, k, q, q);
    for (int k = 0; k < M; ++k)                                                           // R4
        for (int l = 0; l < M; ++l)
            if (l != k) at(pr(k, k), pr(k, l)) += H(k, k, k, l);
    for (int k = 0; k < M; ++k)                                                           // R5
        for (int s = 0; s < M; ++s)
            if (s != k) at(pr(k, s), pr(s, s)) += H(k, s, s, s);
    for (int k = 0; k < M; ++k)                                                           // R6
        for (int q = 0; q < M; ++q)
            for (int l = q + 1; l < M; ++l)
                if (q != k && l != k) at(pr(k, k), pr(q, l)) += H(k, k, q, l);
    for (int k = 0; k < M; ++k)                                                           // R7
        for (int s = k + 1; s < M; ++s)
            for (int q = 0; q < M; ++q)
                if (q != k && q != s) at(pr(k, s), pr(q, q)) += H(k, s, q, q);
    for (int s = 0; s < M; ++s)                                                           // R8
        for (int k = 0; k < M; ++k)
            for (int l = 0; l < M; ++l)
                if (k != s && l != k && l != s) at(pr(k, s), pr(s, l)) += 2.0 * H(k, s, s, l);
    for (int k = 0; k < M; ++k)                                                           // R9
        for (int s = k + 1; s < M; ++s)
            for (int q = 0; q < M; ++q)
                for (int l = q + 1; l < M; ++l) {
                    if (q == k || q == s || l == k || l == s) continue;
                    if (hash_variant)
                        at(pr(k, s), pr(q, l)) += 0.5 * (H(k, s, q, l) + H(s, k, q, l) + H(k, s, l, q) + H(s, k, l, q));
                    else
                        at(pr(k, s), pr(q, l)) += 2.0 * H(k, s, q, l);
                }
    // off-diagonal one-body, folded
    const double f = 1.0 / (N - 1);
    for (int k = 0; k < M; ++k)
        for (int l = 0; l < M; ++l) {
            if (k == l || Ho[k * M + l] == cplx(0.0, 0.0)) continue;
            for (int s = 0; s < M; ++s) at(pr(k, s), pr(s, l)) += f * Ho[k * M + l];
        }
}

}  // namespace mcpi
