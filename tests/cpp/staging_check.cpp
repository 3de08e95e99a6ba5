// Host emulation of the range logic of the TMA-staged pair-creation kernel
// (mcpi_b200/csrc/hpsi.cu, k_pair_create_tma): for blocks of R consecutive
// rows (the last one partial), the rows holding pair a must read a gap-free
// range E[a][lo..hi] (hi - lo + 1 = number of such rows), every range must lie
// inside [0, nc2), and every shared-memory slot a row reads must lie inside
// the block's staged total, which must fit the P*R slots allocated. Uses the
// same header as the kernels. Prints "ok"; exit status 0 on success.
#include <cstdio>
#include <vector>
#include "../../mcpi_b200/csrc/fock.cuh"

using namespace mcpi;

template <int M>
static int check(int N, int R, int stride_blocks)
{
    constexpr int P = M * (M + 1) / 2;
    std::vector<std::vector<uint64_t>> C(N + M + 6, std::vector<uint64_t>(N + M + 6, 0));
    for (size_t a = 0; a < C.size(); ++a) {
        C[a][0] = 1;
        for (size_t b = 1; b <= a; ++b) C[a][b] = C[a - 1][b - 1] + (b <= a - 1 ? C[a - 1][b] : 0);
    }
    const int ws = N + 3;
    std::vector<uint32_t> W((M > 1 ? M - 1 : 1) * ws);
    for (int i = 0; i + 1 < M; ++i)
        for (int p = 0; p < ws; ++p) W[i * ws + p] = (uint32_t)C[p + i][i + 1];
    const uint32_t nc = (uint32_t)C[N + M - 1][N], nc2 = (uint32_t)C[N - 2 + M - 1][N - 2];
    const uint32_t nblocks = (nc + R - 1) / R;
    for (uint32_t b = 0; b < nblocks; b += (b + 1 == nblocks || b + stride_blocks < nblocks) ? stride_blocks : nblocks - 1 - b) {
        std::vector<uint32_t> lo(P, 0xffffffffu), hi(P, 0), cnt(P, 0);
        std::vector<std::vector<uint32_t>> mms(R, std::vector<uint32_t>(P, 0xffffffffu));
        for (int t = 0; t < R; ++t) {
            const uint32_t i = b * R + t;
            if (i >= nc) continue;
            int v[M], Pp[M];
            decode<M>(i, N, nc, W.data(), ws, v, Pp);
            uint32_t A0[M], Am1[M], Am2[M];
            prefix_table<M>(Pp, 0, W.data(), ws, A0);
            prefix_table<M>(Pp, -1, W.data(), ws, Am1);
            prefix_table<M>(Pp, -2, W.data(), ws, Am2);
            const uint32_t base = nc2 - 1u - Am2[M - 1];
            for (int k = 0; k < M; ++k)
                for (int s = k; s < M; ++s) {
                    const bool ok = (s == k) ? (v[k] >= 2) : (v[k] >= 1 && v[s] >= 1);
                    if (!ok) continue;
                    const uint32_t mm = (base - (A0[k] - Am1[k])) - (Am1[s] - Am2[s]);
                    const int a = pair_index(k, s, M);
                    if (mm >= nc2) { printf("index out of range\n"); return 1; }
                    lo[a] = mm < lo[a] ? mm : lo[a];
                    hi[a] = mm > hi[a] ? mm : hi[a];
                    cnt[a]++;
                    mms[t][a] = mm;
                }
        }
        uint32_t total = 0;
        std::vector<uint32_t> off(P);
        for (int a = 0; a < P; ++a) {
            off[a] = total;
            if (lo[a] <= hi[a]) {
                if (hi[a] - lo[a] + 1 != cnt[a]) { printf("range has gaps (block %u pair %d)\n", b, a); return 1; }
                total += hi[a] - lo[a] + 1;
            }
        }
        if (total > (uint32_t)(P * R)) { printf("staging overflow\n"); return 1; }
        for (int t = 0; t < R; ++t)
            for (int a = 0; a < P; ++a)
                if (mms[t][a] != 0xffffffffu) {
                    const uint32_t slot = off[a] + (mms[t][a] - lo[a]);
                    if (slot >= total) { printf("slot outside staged data\n"); return 1; }
                }
    }
    return 0;
}

int main()
{
    int bad = 0;
    bad |= check<10>(16, 128, 97);     // N=16 M=10 (benchmark space), sampled blocks + the last
    bad |= check<10>(20, 128, 4001);   // N=20 M=10
    bad |= check<10>(10, 128, 1);      // N=10 M=10, every block
    bad |= check<11>(14, 64, 2001);
    bad |= check<7>(9, 128, 1);
    bad |= check<9>(12, 128, 37);
    bad |= check<16>(6, 32, 11);
    bad |= check<3>(2, 128, 1);
    bad |= check<2>(5, 128, 1);
    bad |= check<1>(4, 128, 1);
    printf(bad ? "FAILED\n" : "ok\n");
    return bad;
}
