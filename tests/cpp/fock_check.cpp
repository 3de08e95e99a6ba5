// Host check of the device index arithmetic (mcpi_b200/csrc/fock.cuh): for
// every configuration of the given spaces, the prefix-table formulas must agree
// with a brute-force enumeration in the reference's order (index 0 = all
// particles in orbital 0, FockToIndex of configurationsMap.h:273-305), and
// every jump index must stay inside its target space. Prints "ok" or the first
// mismatch; exit status 0 on success. Built and run by tests/test_fock_host.py.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <vector>
#include "../../mcpi_b200/csrc/fock.cuh"

using namespace mcpi;

static std::vector<std::vector<uint64_t>> pascal(int n)
{
    std::vector<std::vector<uint64_t>> C(n + 1, std::vector<uint64_t>(n + 1, 0));
    for (int a = 0; a <= n; ++a) {
        C[a][0] = 1;
        for (int b = 1; b <= a; ++b) C[a][b] = C[a - 1][b - 1] + (b <= a - 1 ? C[a - 1][b] : 0);
    }
    return C;
}

// reference-order index by the reference's own recipe (NC of the remaining particles)
static int64_t ref_index(const std::vector<int> &v, int n, int M, const std::vector<std::vector<uint64_t>> &C)
{
    auto NCf = [&](int nn, int m) -> int64_t { return m <= 0 ? 0 : (int64_t)C[nn + m - 1][nn]; };
    int64_t k = 0;
    for (int i = M - 1; i > 0; --i)
        for (int p = v[i]; p > 0; --p) { k += NCf(n, i); n--; }
    return k;
}

template <int M>
static int check(int N, uint32_t step)
{
    auto C = pascal(N + M + 4);
    const int ws = N + 3;
    std::vector<uint32_t> W((M > 1 ? M - 1 : 1) * ws);
    for (int i = 0; i + 1 < M; ++i)
        for (int p = 0; p < ws; ++p) W[i * ws + p] = (uint32_t)C[p + i][i + 1];
    auto NCf = [&](int n, int m) -> uint32_t { return n < 0 ? 0 : (uint32_t)C[n + m - 1][n]; };
    auto refi = [&](const std::vector<int> &x, int n) { return ref_index(x, n, M, C); };
    const uint32_t nc = NCf(N, M), nc1 = NCf(N - 1, M), nc2 = NCf(N - 2, M);
    // configurations of N, N-1, N-2 particles: decode round trip + every jump
    for (int d = 0; d < 3 && N - d >= 0; ++d) {
        const int n = N - d;
        const uint32_t ncn = NCf(n, M);
        for (uint64_t ii = 0; ii < ncn; ii += (d == 0 ? step : step / 2 + 1)) {
            const uint32_t i = (uint32_t)ii;
            int v[M], P[M];
            decode<M>(i, n, ncn, W.data(), ws, v, P);
            std::vector<int> vv(v, v + M);
            int tot = 0;
            for (int t = 0; t < M; ++t) {
                if (v[t] < 0) { printf("negative occupation\n"); return 1; }
                tot += v[t];
            }
            if (tot != n || refi(vv, n) != i) { printf("decode mismatch n=%d M=%d i=%u\n", n, M, i); return 1; }
            uint32_t A0[M], Am1[M], Am2[M], Ap1[M], Ap2[M];
            prefix_table<M>(P, 0, W.data(), ws, A0);
            prefix_table<M>(P, -1, W.data(), ws, Am1);
            prefix_table<M>(P, -2, W.data(), ws, Am2);
            prefix_table<M>(P, 1, W.data(), ws, Ap1);
            prefix_table<M>(P, 2, W.data(), ws, Ap2);
            if (d == 0) {
                for (int k = 0; k < M; ++k)
                    for (int s = k; s < M; ++s) {
                        bool ok = s == k ? v[k] >= 2 : (v[k] >= 1 && v[s] >= 1);
                        if (!ok) continue;
                        std::vector<int> w = vv; w[k]--; w[s]--;
                        uint32_t m = idx_remove2(nc2, A0, Am1, Am2, k, s, M);
                        if (m >= nc2 || refi(w, N - 2) != m) { printf("remove2 mismatch\n"); return 1; }
                    }
                for (int k = 0; k < M; ++k) {
                    if (v[k] < 1) continue;
                    std::vector<int> w = vv; w[k]--;
                    uint32_t m = idx_remove1(nc1, A0, Am1, k, M);
                    if (m >= nc1 || refi(w, N - 1) != m) { printf("remove1 mismatch\n"); return 1; }
                    for (int l = 0; l < M; ++l) {
                        std::vector<int> x = w; x[l]++;
                        uint32_t j = idx_move1(nc, A0, Am1, Ap1, k, l, M);
                        if (j >= nc || refi(x, N) != j) { printf("move1 mismatch k=%d l=%d\n", k, l); return 1; }
                    }
                }
            } else if (d == 1) {
                for (int l = 0; l < M; ++l) {
                    std::vector<int> x = vv; x[l]++;
                    uint32_t j = idx_add1(nc, A0, Ap1, l, M);
                    if (j >= nc || refi(x, N) != j) { printf("add1 mismatch\n"); return 1; }
                }
            } else {
                for (int q = 0; q < M; ++q)
                    for (int l = q; l < M; ++l) {
                        std::vector<int> x = vv; x[q]++; x[l]++;
                        uint32_t j = idx_add2(nc, A0, Ap1, Ap2, q, l, M);
                        if (j >= nc || refi(x, N) != j) { printf("add2 mismatch\n"); return 1; }
                    }
            }
        }
    }
    return 0;
}

int main(int argc, char **argv)
{
    const bool large = argc > 1;
    int bad = 0;
    for (int N = 0; N <= 7; ++N) {
        bad |= check<1>(N, 1); bad |= check<2>(N, 1); bad |= check<3>(N, 1); bad |= check<4>(N, 1);
        bad |= check<5>(N, 1); bad |= check<6>(N, 1);
    }
    for (int N = 0; N <= 6; ++N) { bad |= check<7>(N, 1); bad |= check<9>(N, 1); bad |= check<10>(N, 1); bad |= check<11>(N, 1); }
    for (int N = 0; N <= 4; ++N) { bad |= check<13>(N, 1); bad |= check<16>(N, 1); }
    if (large) {   // the benchmark and batch spaces, sampled rows
        bad |= check<10>(16, 101); bad |= check<10>(20, 997); bad |= check<11>(14, 97);
        bad |= check<7>(14, 7); bad |= check<9>(14, 31); bad |= check<16>(9, 499);
    }
    printf(bad ? "FAILED\n" : "ok\n");
    return bad;
}
