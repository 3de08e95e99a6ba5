/* mcpi CPU oracle: a plain-C restatement of the reference's hot path.
 *
 * TEST INFRASTRUCTURE ONLY. tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs load this library (oracle/liborc.so) as the
 * checker or as the timed CPU baseline. The product (mcpi_b200/) never links,
 * imports or calls it.
 *
 * What is restated, and from where (file:line in the reference project):
 *   orc_nc / orc_ncmat           configurationsMap.h:145-234  NC, setupNCmat
 *   orc_index_to_fock            configurationsMap.h:238-269  IndexToFock
 *   orc_fock_to_index            configurationsMap.h:273-305  FockToIndex
 *   orc_setup_focks              configurationsMap.h:309-344  setupFocks
 *   orc_one_one_map              configurationsMap.h:348-417  OneOneMap
 *   orc_one_two_* (count, map)   configurationsMap.h:617-762  allocOneTwoMap, OneTwoMap
 *   orc_two_two_* (count, map)   configurationsMap.h:421-613  allocTwoTwoMap, TwoTwoMap
 *   orc_apply_h                  hamiltonianMatrix.h:31-425 (plain), :431-887 (_X),
 *                                :891-1425 (_XX), :1431-1970 (_omp = _XX over threads)
 *   orc_obrho                    onebodyMatrix.h:190-251      OBrho_XM
 *   orc_density_generic / _rows  definition of rho1/rho2 in onebodyMatrix.h:20-30 and
 *                                twobodyMatrix.h:20-36, evaluated term by term for a
 *                                bra/ket pair (also gives the transition densities)
 *   orc_apply_h_generic          H = sum Ho a+a + 1/2 sum Hint a+a+aa, unfolded
 *   orc_lieb_ho / orc_lieb_hint  groundStateLieb.c:129-213     setupHo, setupHint
 *   orc_perf_inputs              performanceTest.c:169-219     deterministic C, Ho, Hint
 *   orc_lanczos / orc_ground     groundStateLieb.c:217-471     lanczos, ground
 *
 * Differences from the reference, all deliberate: strides and map offsets are
 * 64-bit (the reference's int32 arithmetic aborts at N=16,M=10), H.psi takes a
 * row range [row0,row1) and an OpenMP thread count so that a bounded sample of
 * a large configuration can be timed, and errors are return codes, not exit().
 * Inside each row the terms are accumulated in the reference's loop order and
 * with the reference's expression shapes, so results are bit-identical to the
 * reference's when both are compiled with the same compiler flags.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "shim/mkl.h"

typedef double complex zc;

/* ------------------------------------------------------------------ */
/* combinatorics                                                      */
/* ------------------------------------------------------------------ */

/* NC(N,M) = C(N+M-1, N): configurations of N bosons in M orbitals
 * (configurationsMap.h:145-202). Exact in 64 bits; -1 when it does not fit. */
int64_t orc_nc(int N, int M)
{
    if (N < 0 || M < 1) return 0;
    int64_t n = (int64_t)N + M - 1;
    int64_t k = (M - 1 < N) ? (M - 1) : N;
    __int128 r = 1;
    for (int64_t i = 1; i <= k; i++) {
        r = r * (n - k + i) / i;
        if (r > INT64_MAX) return -1;
    }
    return (int64_t)r;
}

/* NCmat[n + (N+1)*m] = NC(n,m), row m=0 -> 0, m=1 -> 1
 * (configurationsMap.h:206-234). */
void orc_ncmat(int N, int M, int32_t *t)
{
    for (int n = 0; n <= N; n++) {
        t[n + (N + 1) * 0] = 0;
        if (M >= 1) t[n + (N + 1) * 1] = 1;
        for (int m = 2; m <= M; m++) t[n + (N + 1) * m] = (int32_t)orc_nc(n, m);
    }
}

typedef struct {
    int N, M;
    int64_t nc;
    int64_t *t; /* t[n + (N+1)*m] = NC(n,m), 64-bit copy of NCmat */
} space_t;

static int space_init(space_t *sp, int N, int M)
{
    sp->N = N;
    sp->M = M;
    sp->nc = orc_nc(N, M);
    sp->t = (int64_t *)malloc(sizeof(int64_t) * (N + 1) * (M + 1));
    if (!sp->t) return -1;
    for (int n = 0; n <= N; n++) {
        sp->t[n] = 0;
        if (M >= 1) sp->t[n + (N + 1)] = 1;
        for (int m = 2; m <= M; m++) sp->t[n + (N + 1) * m] = orc_nc(n, m);
    }
    return 0;
}

static void space_free(space_t *sp) { free(sp->t); }

/* Greedy decode of an index into occupations (configurationsMap.h:238-269):
 * from the top orbital down, place one particle at the highest orbital whose
 * cost NC(n,m) still fits in the remaining index, subtract, repeat; whatever
 * is left when the index reaches 0 goes to orbital 0. */
static void index_to_fock(const space_t *sp, int64_t k, int *v)
{
    int N = sp->N, M = sp->M, m = M - 1;
    for (int i = 0; i < M; i++) v[i] = 0;
    while (k > 0) {
        while (k - sp->t[N + (sp->N + 1) * m] < 0) m--;
        k -= sp->t[N + (sp->N + 1) * m];
        v[m] += 1;
        N -= 1;
    }
    if (N > 0) v[0] += N;
}

/* Encode occupations into the index (configurationsMap.h:273-305): empty the
 * orbitals from the top, each particle removed from orbital i adding
 * NC(n_remaining, i). */
static int64_t fock_to_index(const space_t *sp, const int *v)
{
    int64_t k = 0;
    int n = sp->N;
    for (int i = sp->M - 1; i > 0; i--)
        for (int p = v[i]; p > 0; p--) {
            k += sp->t[n + (sp->N + 1) * i];
            n -= 1;
        }
    return k;
}

void orc_index_to_fock(int64_t k, int N, int M, int32_t *v)
{
    space_t sp;
    int tmp[64];
    if (space_init(&sp, N, M)) return;
    index_to_fock(&sp, k, tmp);
    for (int i = 0; i < M; i++) v[i] = tmp[i];
    space_free(&sp);
}

int64_t orc_fock_to_index(int N, int M, const int32_t *v)
{
    space_t sp;
    int tmp[64];
    if (space_init(&sp, N, M)) return -1;
    for (int i = 0; i < M; i++) tmp[i] = v[i];
    int64_t k = fock_to_index(&sp, tmp);
    space_free(&sp);
    return k;
}

/* IF[j + k*M] = occupation of orbital j in configuration k
 * (configurationsMap.h:309-344). */
int orc_setup_focks(int N, int M, int32_t *IF, int nthreads)
{
    space_t sp;
    if (M > 64 || space_init(&sp, N, M)) return -1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t k = 0; k < sp.nc; k++) {
        int v[64];
        index_to_fock(&sp, k, v);
        for (int j = 0; j < M; j++) IF[j + k * M] = v[j];
    }
    space_free(&sp);
    return 0;
}

/* One-jump map (configurationsMap.h:348-417):
 * Map[i + k*nc + l*M*nc] = index of v - e_k + e_l, -1 when v_k = 0. */
int orc_one_one_map(int N, int M, const int32_t *IF, int32_t *Map, int nthreads)
{
    space_t sp;
    if (M > 64 || space_init(&sp, N, M)) return -1;
    int64_t nc = sp.nc;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < nc; i++) {
        int v[64];
        for (int q = 0; q < M; q++) v[q] = IF[q + M * i];
        for (int k = 0; k < M; k++)
            for (int l = 0; l < M; l++) {
                int64_t at = i + k * nc + (int64_t)l * M * nc;
                if (v[k] < 1) { Map[at] = -1; continue; }
                v[k] -= 1;
                v[l] += 1;
                Map[at] = (int32_t)fock_to_index(&sp, v);
                v[k] += 1;
                v[l] -= 1;
            }
    }
    space_free(&sp);
    return 0;
}

/* Chunk counts of the two-particle maps. A configuration owns one chunk of
 * M*M entries per orbital with v_k >= 2 (one-orbital map, allocOneTwoMap,
 * configurationsMap.h:617-664) or per orbital pair k<s with v_k,v_s >= 1
 * (two-orbital map, allocTwoTwoMap, configurationsMap.h:421-474).
 * stride[i] = M*M * (chunks of all configurations before i), 64-bit.
 * Returns the total number of chunks. */
static int chunks_of(const int32_t *row, int M, int two_orbital)
{
    int c = 0;
    if (!two_orbital) {
        for (int k = 0; k < M; k++) c += (row[k] >= 2);
    } else {
        for (int k = 0; k < M; k++) {
            if (row[k] < 1) continue;
            for (int s = k + 1; s < M; s++) c += (row[s] >= 1);
        }
    }
    return c;
}

static int64_t two_map_strides(int64_t nc, int M, const int32_t *IF,
                               int64_t *stride, int two_orbital)
{
    int64_t total = 0;
    for (int64_t i = 0; i < nc; i++) {
        if (stride) stride[i] = total * M * M;
        total += chunks_of(IF + i * M, M, two_orbital);
    }
    return total;
}

int64_t orc_one_two_strides(int N, int M, const int32_t *IF, int64_t *stride)
{
    return two_map_strides(orc_nc(N, M), M, IF, stride, 0);
}

int64_t orc_two_two_strides(int N, int M, const int32_t *IF, int64_t *stride)
{
    return two_map_strides(orc_nc(N, M), M, IF, stride, 1);
}

/* One-orbital double jump (configurationsMap.h:668-762):
 * MapOT[stride[i] + c*M*M + (l + q*M)] = index of v - 2e_k + e_l + e_q, with
 * c the rank of k among the orbitals of v holding at least two particles. */
int orc_one_two_map(int N, int M, const int32_t *IF, const int64_t *stride,
                    int32_t *Map, int nthreads)
{
    space_t sp;
    if (M > 64 || space_init(&sp, N, M)) return -1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < sp.nc; i++) {
        int v[64];
        int64_t c = 0;
        for (int q = 0; q < M; q++) v[q] = IF[q + M * i];
        for (int k = 0; k < M; k++) {
            if (v[k] < 2) continue;
            int64_t base = stride[i] + c * M * M;
            for (int l = 0; l < M; l++)
                for (int q = 0; q < M; q++) {
                    v[k] -= 2;
                    v[l] += 1;
                    v[q] += 1;
                    Map[base + l + q * M] = (int32_t)fock_to_index(&sp, v);
                    v[k] += 2;
                    v[l] -= 1;
                    v[q] -= 1;
                }
            c++;
        }
    }
    space_free(&sp);
    return 0;
}

/* Two-orbital double jump (configurationsMap.h:478-613):
 * MapTT[stride[i] + c*M*M + (l + q*M)] = index of v - e_k - e_s + e_l + e_q,
 * c the lexicographic rank of the occupied pair (k<s). */
int orc_two_two_map(int N, int M, const int32_t *IF, const int64_t *stride,
                    int32_t *Map, int nthreads)
{
    space_t sp;
    if (M > 64 || space_init(&sp, N, M)) return -1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < sp.nc; i++) {
        int v[64];
        int64_t c = 0;
        for (int q = 0; q < M; q++) v[q] = IF[q + M * i];
        for (int k = 0; k < M; k++) {
            if (v[k] < 1) continue;
            for (int s = k + 1; s < M; s++) {
                if (v[s] < 1) continue;
                int64_t base = stride[i] + c * M * M;
                for (int l = 0; l < M; l++)
                    for (int q = 0; q < M; q++) {
                        v[k] -= 1;
                        v[s] -= 1;
                        v[l] += 1;
                        v[q] += 1;
                        Map[base + l + q * M] = (int32_t)fock_to_index(&sp, v);
                        v[k] += 1;
                        v[s] += 1;
                        v[l] -= 1;
                        v[q] -= 1;
                    }
                c++;
            }
        }
    }
    space_free(&sp);
    return 0;
}

/* ------------------------------------------------------------------ */
/* H.psi                                                              */
/* ------------------------------------------------------------------ */

enum { ORC_PLAIN = 0, ORC_X = 1, ORC_XX = 2 };

typedef struct {
    space_t sp;
    int mode;
    const int32_t *IF, *Map, *MapOT, *MapTT;
    const int64_t *sOT, *sTT;
} hctx_t;

/* index of v - e_k + e_l */
static inline int64_t jmp1(const hctx_t *h, int64_t i, int *v, int k, int l)
{
    if (h->Map && h->mode != ORC_PLAIN)
        return h->Map[i + k * h->sp.nc + (int64_t)l * h->sp.M * h->sp.nc];
    v[k] -= 1;
    v[l] += 1;
    int64_t j = fock_to_index(&h->sp, v);
    v[k] += 1;
    v[l] -= 1;
    return j;
}

/* index of v - 2e_k + e_q + e_l. Map lookup as hamiltonianMatrix.h:1021-1027. */
static inline int64_t jmpOT(const hctx_t *h, int64_t i, int *v, int k, int q, int l)
{
    int M = h->sp.M;
    if (h->MapOT && h->mode != ORC_PLAIN) {
        int64_t c = 0;
        for (int j = 0; j < k; j++) c += (v[j] > 1);
        return h->MapOT[h->sOT[i] + c * M * M + q + (int64_t)l * M];
    }
    v[k] -= 2;
    v[q] += 1;
    v[l] += 1;
    int64_t j = fock_to_index(&h->sp, v);
    v[k] += 2;
    v[q] -= 1;
    v[l] -= 1;
    return j;
}

/* index of v - e_k - e_s + e_q + e_l (k<s). Map lookup as
 * hamiltonianMatrix.h:1206-1222; only the all-maps variant uses MapTT. */
static inline int64_t jmpTT(const hctx_t *h, int64_t i, int *v, int k, int s, int q, int l)
{
    int M = h->sp.M;
    if (h->MapTT && h->mode == ORC_XX) {
        int64_t c = 0;
        for (int a = 0; a < k; a++)
            for (int b = a + 1; b < M; b++) c += (v[a] > 0 && v[b] > 0);
        for (int b = k + 1; b < s; b++) c += (v[b] > 0);
        return h->MapTT[h->sTT[i] + c * M * M + q + (int64_t)l * M];
    }
    v[k] -= 1;
    v[s] -= 1;
    v[q] += 1;
    v[l] += 1;
    int64_t j = fock_to_index(&h->sp, v);
    v[k] += 1;
    v[s] += 1;
    v[q] -= 1;
    v[l] -= 1;
    return j;
}

/* One row of out = H.C in the reference's rule order (hamiltonianMatrix.h:
 * 938-1421 for the map variants; :70-422 for the plain one, which differs
 * only in Rule 9, summed over all ordered pairs with weight 1). */
static zc apply_row(const hctx_t *h, int64_t i, const zc *C, const zc *Ho,
                    const zc *Hint)
{
    int M = h->sp.M, M2 = M * M, M3 = M * M * M;
    int v[64];
    double sqrtOf;
    zc w = 0, z = 0;
    int64_t j;
    for (int k = 0; k < M; k++) v[k] = h->IF[k + i * M];

    for (int k = 0; k < M; k++) { /* one-body */
        if (v[k] < 1) continue;
        w = w + Ho[k * M + k] * v[k] * C[i];
        for (int l = 0; l < M; l++) {
            if (l == k) continue;
            sqrtOf = sqrt((double)v[k] * (v[l] + 1));
            j = jmp1(h, i, v, k, l);
            w = w + Ho[k * M + l] * sqrtOf * C[j];
        }
    }
    for (int k = 0; k < M; k++) { /* Rule 1 */
        sqrtOf = v[k] * (v[k] - 1);
        z += Hint[k + M * k + M2 * k + M3 * k] * C[i] * sqrtOf;
    }
    for (int k = 0; k < M; k++) { /* Rule 2 */
        if (v[k] < 1) continue;
        for (int s = k + 1; s < M; s++) {
            sqrtOf = v[k] * v[s];
            z += 4 * Hint[k + s * M + k * M2 + s * M3] * sqrtOf * C[i];
        }
    }
    for (int k = 0; k < M; k++) { /* Rule 3 */
        if (v[k] < 2) continue;
        for (int q = 0; q < M; q++) {
            if (q == k) continue;
            sqrtOf = sqrt((double)(v[k] - 1) * v[k] * (v[q] + 1) * (v[q] + 2));
            j = jmpOT(h, i, v, k, q, q);
            z += Hint[k + k * M + q * M2 + q * M3] * C[j] * sqrtOf;
        }
    }
    for (int k = 0; k < M; k++) { /* Rule 4 */
        if (v[k] < 2) continue;
        for (int l = 0; l < M; l++) {
            if (l == k) continue;
            sqrtOf = (v[k] - 1) * sqrt((double)v[k] * (v[l] + 1));
            j = jmp1(h, i, v, k, l);
            z += 2 * Hint[k + k * M + k * M2 + l * M3] * C[j] * sqrtOf;
        }
    }
    for (int k = 0; k < M; k++) { /* Rule 5 */
        if (v[k] < 1) continue;
        for (int s = 0; s < M; s++) {
            if (s == k || v[s] < 1) continue;
            sqrtOf = v[s] * sqrt((double)v[k] * (v[s] + 1));
            j = jmp1(h, i, v, k, s);
            z += 2 * Hint[k + s * M + s * M2 + s * M3] * C[j] * sqrtOf;
        }
    }
#define R6_TERM                                                            \
    do {                                                                   \
        sqrtOf = sqrt((double)v[k] * (v[k] - 1) * (v[q] + 1) * (v[l] + 1)); \
        j = jmpOT(h, i, v, k, q, l);                                       \
        z += 2 * Hint[k + k * M + q * M2 + l * M3] * C[j] * sqrtOf;        \
    } while (0)
    for (int k = 0; k < M; k++) { /* Rule 6.0 */
        if (v[k] < 2) continue;
        for (int q = k + 1; q < M; q++)
            for (int l = q + 1; l < M; l++) R6_TERM;
    }
    for (int q = 0; q < M; q++) /* Rule 6.1 */
        for (int k = q + 1; k < M; k++) {
            if (v[k] < 2) continue;
            for (int l = k + 1; l < M; l++) R6_TERM;
        }
    for (int q = 0; q < M; q++) /* Rule 6.2 */
        for (int l = q + 1; l < M; l++)
            for (int k = l + 1; k < M; k++) {
                if (v[k] < 2) continue;
                R6_TERM;
            }
#undef R6_TERM
#define R7_TERM                                                               \
    do {                                                                      \
        sqrtOf = sqrt((double)v[k] * v[s] * (v[q] + 1) * (v[q] + 2));         \
        j = jmpTT(h, i, v, k, s, q, q);                                       \
        z += 2 * Hint[k + s * M + q * M2 + q * M3] * C[j] * sqrtOf;           \
    } while (0)
    for (int q = 0; q < M; q++) /* Rule 7.0 */
        for (int k = q + 1; k < M; k++) {
            if (v[k] < 1) continue;
            for (int s = k + 1; s < M; s++) {
                if (v[s] < 1) continue;
                R7_TERM;
            }
        }
    for (int k = 0; k < M; k++) { /* Rule 7.1 */
        if (v[k] < 1) continue;
        for (int q = k + 1; q < M; q++)
            for (int s = q + 1; s < M; s++) {
                if (v[s] < 1) continue;
                R7_TERM;
            }
    }
    for (int k = 0; k < M; k++) { /* Rule 7.2 */
        if (v[k] < 1) continue;
        for (int s = k + 1; s < M; s++) {
            if (v[s] < 1) continue;
            for (int q = s + 1; q < M; q++) R7_TERM;
        }
    }
#undef R7_TERM
    for (int s = 0; s < M; s++) { /* Rule 8 */
        if (v[s] < 1) continue;
        for (int k = 0; k < M; k++) {
            if (v[k] < 1 || k == s) continue;
            for (int l = 0; l < M; l++) {
                if (l == k || l == s) continue;
                sqrtOf = v[s] * sqrt((double)v[k] * (v[l] + 1));
                j = jmp1(h, i, v, k, l);
                z += 4 * Hint[k + s * M + s * M2 + l * M3] * C[j] * sqrtOf;
            }
        }
    }
    if (h->mode == ORC_PLAIN) { /* Rule 9, hash-only variant */
        for (int k = 0; k < M; k++) {
            if (v[k] < 1) continue;
            for (int s = 0; s < M; s++) {
                if (v[s] < 1 || s == k) continue;
                for (int q = 0; q < M; q++) {
                    if (q == s || q == k) continue;
                    for (int l = 0; l < M; l++) {
                        if (l == k || l == s || l == q) continue;
                        sqrtOf = sqrt((double)v[k] * v[s] * (v[q] + 1) * (v[l] + 1));
                        v[k] -= 1;
                        v[s] -= 1;
                        v[q] += 1;
                        v[l] += 1;
                        j = fock_to_index(&h->sp, v);
                        v[k] += 1;
                        v[s] += 1;
                        v[q] -= 1;
                        v[l] -= 1;
                        z += Hint[k + s * M + q * M2 + l * M3] * C[j] * sqrtOf;
                    }
                }
            }
        }
    } else { /* Rule 9, map variants */
        for (int k = 0; k < M; k++) {
            if (v[k] < 1) continue;
            for (int s = k + 1; s < M; s++) {
                if (v[s] < 1) continue;
                for (int q = 0; q < M; q++) {
                    if (q == s || q == k) continue;
                    for (int l = q + 1; l < M; l++) {
                        if (l == k || l == s) continue;
                        sqrtOf = sqrt((double)v[k] * v[s] * (v[q] + 1) * (v[l] + 1));
                        j = jmpTT(h, i, v, k, s, q, l);
                        z += 4 * Hint[k + s * M + q * M2 + l * M3] * C[j] * sqrtOf;
                    }
                }
            }
        }
    }
    return w + 0.5 * z;
}

/* out[i] for i in [row0,row1). mode: 0 plain (hash only), 1 _X (Map, MapOT,
 * hash for rules 7/9), 2 _XX (all maps). Any map pointer may be NULL, in
 * which case that lookup is done with the hash (same indices). Ho is flat
 * row-major: Ho[k*M + l] is the reference's Ho[k][l]. */
int orc_apply_h(int N, int M, int mode, const int32_t *IF, const int32_t *Map,
                const int32_t *MapOT, const int64_t *strideOT, const int32_t *MapTT,
                const int64_t *strideTT, const zc *C, const zc *Ho, const zc *Hint,
                zc *out, int64_t row0, int64_t row1, int nthreads)
{
    hctx_t h;
    if (M > 64 || space_init(&h.sp, N, M)) return -1;
    h.mode = mode;
    h.IF = IF;
    h.Map = Map;
    h.MapOT = MapOT;
    h.MapTT = MapTT;
    h.sOT = strideOT;
    h.sTT = strideTT;
    if (row1 > h.sp.nc) row1 = h.sp.nc;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
    for (int64_t i = row0; i < row1; i++) out[i] = apply_row(&h, i, C, Ho, Hint);
    space_free(&h.sp);
    return 0;
}

/* ------------------------------------------------------------------ */
/* densities                                                          */
/* ------------------------------------------------------------------ */

/* rho[k*M + l] = <a+_k a_l>, OBrho_XM order (onebodyMatrix.h:190-251):
 * diagonal from |C_i|^2 v_k, upper triangle by a reduction over rows,
 * lower triangle as the conjugate. Map may be NULL (hash). */
int orc_obrho(int N, int M, const int32_t *IF, const int32_t *Map, const zc *C, zc *rho)
{
    hctx_t h;
    if (M > 64 || space_init(&h.sp, N, M)) return -1;
    h.mode = ORC_XX;
    h.IF = IF;
    h.Map = Map;
    int64_t nc = h.sp.nc;
    for (int k = 0; k < M; k++) {
        zc RHO = 0;
        for (int64_t i = 0; i < nc; i++) {
            double mod2 = creal(C[i]) * creal(C[i]) + cimag(C[i]) * cimag(C[i]);
            RHO = RHO + mod2 * IF[k + i * M];
        }
        rho[k * M + k] = RHO;
        for (int l = k + 1; l < M; l++) {
            RHO = 0;
            for (int64_t i = 0; i < nc; i++) {
                int v[64];
                int vk = IF[k + M * i];
                if (vk < 1) continue;
                int vl = IF[l + M * i];
                for (int a = 0; a < M; a++) v[a] = IF[a + M * i];
                int64_t j = jmp1(&h, i, v, k, l);
                RHO += conj(C[i]) * C[j] * sqrt((double)(vl + 1) * vk);
            }
            rho[k * M + l] = RHO;
            rho[l * M + k] = conj(RHO);
        }
    }
    space_free(&h.sp);
    return 0;
}

/* Densities by definition, for a bra phi and a ket psi:
 *   t1[k + l*M]               = <phi| a+_k a_l |psi>            (order 1)
 *   t2[k + s*M + q*M^2 + l*M^3] = <phi| a+_k a+_s a_q a_l |psi>  (order 2)
 * (index conventions of onebodyMatrix.h / twobodyMatrix.h; with phi = psi
 * these are rho1 and rho2). Every entry is reduced: no symmetry fill, so the
 * result is valid when phi != psi. Only ket rows i in [row0, row1) are summed
 * (the whole space: 0, nc), i.e. the result is <phi| ... |psi_S> with psi_S
 * the ket restricted to those rows. Cost (row1-row0)*M^4*O(M). Rows are
 * split into nthreads fixed chunks whose partial sums are added in chunk
 * order. */
static void density_rows(const space_t *sp, int order, const zc *phi, const zc *psi, zc *t, int64_t r0,
                         int64_t r1)
{
    int M = sp->M;
    int64_t M2 = (int64_t)M * M, M3 = M2 * M;
    int v[64];
    for (int64_t i = r0; i < r1; i++) {
        index_to_fock(sp, i, v);
        if (order == 1) {
            for (int l = 0; l < M; l++) {
                if (v[l] < 1) continue;
                double f1 = sqrt((double)v[l]);
                v[l]--;
                for (int k = 0; k < M; k++) {
                    double f = f1 * sqrt((double)(v[k] + 1));
                    v[k]++;
                    int64_t j = fock_to_index(sp, v);
                    v[k]--;
                    t[k + l * M] += conj(phi[j]) * psi[i] * f;
                }
                v[l]++;
            }
        } else {
            for (int l = 0; l < M; l++) {
                if (v[l] < 1) continue;
                double fl = sqrt((double)v[l]);
                v[l]--;
                for (int q = 0; q < M; q++) {
                    if (v[q] < 1) continue;
                    double fq = sqrt((double)v[q]);
                    v[q]--;
                    for (int s = 0; s < M; s++) {
                        double fs = sqrt((double)(v[s] + 1));
                        v[s]++;
                        for (int k = 0; k < M; k++) {
                            double fk = sqrt((double)(v[k] + 1));
                            v[k]++;
                            int64_t j = fock_to_index(sp, v);
                            v[k]--;
                            t[k + s * M + q * M2 + l * M3] += conj(phi[j]) * psi[i] * (fl * fq * fs * fk);
                        }
                        v[s]--;
                    }
                    v[q]++;
                }
                v[l]++;
            }
        }
    }
}

int orc_density_rows(int N, int M, int order, const zc *phi, const zc *psi, zc *t, int64_t row0, int64_t row1,
                     int nthreads)
{
    space_t sp;
    if (M > 64 || space_init(&sp, N, M)) return -1;
    if (row0 < 0 || row1 > sp.nc || row0 > row1) {
        space_free(&sp);
        return -1;
    }
    int64_t M2 = (int64_t)M * M;
    int64_t nout = order == 1 ? M2 : M2 * M2;
    if (nthreads < 1) nthreads = 1;
    zc *part = (zc *)calloc((size_t)nthreads * nout, sizeof(zc));
    if (!part) {
        space_free(&sp);
        return -1;
    }
    int64_t n = row1 - row0;
#pragma omp parallel for schedule(static, 1) num_threads(nthreads)
    for (int c = 0; c < nthreads; c++)
        density_rows(&sp, order, phi, psi, part + (int64_t)c * nout, row0 + n * c / nthreads,
                     row0 + n * (c + 1) / nthreads);
    for (int64_t x = 0; x < nout; x++) {
        zc z = 0;
        for (int c = 0; c < nthreads; c++) z += part[(int64_t)c * nout + x];
        t[x] = z;
    }
    free(part);
    space_free(&sp);
    return 0;
}

int orc_density_generic(int N, int M, int order, const zc *phi, const zc *psi, zc *t)
{
    space_t sp;
    if (M > 64 || space_init(&sp, N, M)) return -1;
    int64_t M2 = (int64_t)M * M;
    int64_t nout = order == 1 ? M2 : M2 * M2;
    for (int64_t x = 0; x < nout; x++) t[x] = 0;
    density_rows(&sp, order, phi, psi, t, 0, sp.nc);
    space_free(&sp);
    return 0;
}

/* out = H psi with H = sum_kl Ho[k][l] a+_k a_l + 1/2 sum Hint[k,s,q,l]
 * a+_k a+_s a_q a_l, every ordered index tuple summed (no folding). For a
 * Hint with the full bosonic 8-fold symmetry this equals every reference
 * variant; it is the operator whose derivatives the adjoint tests check. */
int orc_apply_h_generic(int N, int M, const zc *Ho, const zc *Hint, const zc *psi, zc *out)
{
    space_t sp;
    if (M > 64 || space_init(&sp, N, M)) return -1;
    int64_t nc = sp.nc, M2 = (int64_t)M * M, M3 = M2 * M;
    int v[64];
    for (int64_t i = 0; i < nc; i++) out[i] = 0;
    for (int64_t i = 0; i < nc; i++) {
        index_to_fock(&sp, i, v);
        for (int l = 0; l < M; l++) {
            if (v[l] < 1) continue;
            double fl = sqrt((double)v[l]);
            v[l]--;
            for (int k = 0; k < M; k++) {
                double fk = sqrt((double)(v[k] + 1));
                v[k]++;
                out[fock_to_index(&sp, v)] += Ho[k * M + l] * psi[i] * (fl * fk);
                v[k]--;
            }
            for (int q = 0; q < M; q++) {
                if (v[q] < 1) continue;
                double fq = sqrt((double)v[q]);
                v[q]--;
                for (int s = 0; s < M; s++) {
                    double fs = sqrt((double)(v[s] + 1));
                    v[s]++;
                    for (int k = 0; k < M; k++) {
                        double fk = sqrt((double)(v[k] + 1));
                        v[k]++;
                        out[fock_to_index(&sp, v)] +=
                            0.5 * Hint[k + s * M + q * M2 + l * M3] * psi[i] * (fl * fq * fs * fk);
                        v[k]--;
                    }
                    v[s]--;
                }
                v[q]++;
            }
            v[l]++;
        }
    }
    space_free(&sp);
    return 0;
}

/* ------------------------------------------------------------------ */
/* inputs                                                             */
/* ------------------------------------------------------------------ */

#define ORC_PI 3.141592653589793

/* Plane waves on a ring of length L, k_n = 2 pi (n - M/2)/L:
 * Ho = diag(k_n^2/2) (groundStateLieb.c:129-155); Hint = g wherever momentum
 * is conserved, n + s = q + l in units of 2 pi/L (groundStateLieb.c:159-213). */
void orc_lieb_ho(int M, double L, zc *Ho)
{
    for (int n = 0; n < M; n++) {
        double k = 2 * ORC_PI * (n - M / 2) / L;
        for (int j = 0; j < M; j++) Ho[n * M + j] = 0.0;
        Ho[n * M + n] = 0.5 * k * k;
    }
}

void orc_lieb_hint(int M, double g, zc *Hint)
{
    int M2 = M * M, M3 = M2 * M;
    for (int n = 0; n < M; n++)
        for (int s = 0; s < M; s++)
            for (int q = 0; q < M; q++)
                for (int l = 0; l < M; l++) {
                    int nk = n - M / 2, sk = s - M / 2, qk = q - M / 2, lk = l - M / 2;
                    Hint[n + s * M + q * M2 + l * M3] = (lk + qk - sk - nk == 0) ? g : 0.0;
                }
}

/* Deterministic benchmark inputs of performanceTest.c:169-219. */
void orc_perf_inputs(int N, int M, zc *C, zc *Ho, zc *Hint)
{
    int64_t nc = orc_nc(N, M);
    double sum = 0.0;
    for (int64_t i = 0; i < nc; i++) {
        C[i] = sin(20 * ((double)i) / nc) * (i % 13) + ((i % 8) - (i % 3)) * I;
        sum = sum + creal(C[i]) * creal(C[i]) + cimag(C[i]) * cimag(C[i]);
    }
    for (int64_t i = 0; i < nc; i++) C[i] = C[i] / sqrt(sum);
    for (int i = 0; i < M; i++) {
        Ho[i * M + i] = (i % 4) - 1;
        for (int j = i + 1; j < M; j++) {
            Ho[i * M + j] = i * (j % 3) - (i % 4) + 5 * (j % 2) - I * (4.123 * i / (j + 1));
            Ho[j * M + i] = conj(Ho[i * M + j]);
        }
    }
    int64_t M2 = (int64_t)M * M, M3 = M2 * M;
    for (int64_t i = 0; i < M2 * M2; i++) Hint[i] = 1.234;
    for (int i = 0; i < M; i++)
        for (int j = i + 1; j < M; j++)
            for (int q = 0; q < M; q++) {
                if (q == i || q == j) continue;
                for (int l = q + 1; l < M; l++) {
                    if (l == i || l == j) continue;
                    zc z = i - 2 + 10 * (j % (i + 1)) - q * l;
                    z = z + I * ((double)i * q - j * l) / M;
                    Hint[i + j * M + q * M2 + l * M3] = z;
                    Hint[i + j * M + l * M2 + q * M3] = z;
                    Hint[j + i * M + l * M2 + q * M3] = z;
                    Hint[j + i * M + q * M2 + l * M3] = z;
                    Hint[q + l * M + i * M2 + j * M3] = conj(z);
                    Hint[q + l * M + j * M2 + i * M3] = conj(z);
                    Hint[l + q * M + i * M2 + j * M3] = conj(z);
                    Hint[l + q * M + j * M2 + i * M3] = conj(z);
                }
            }
}

/* ------------------------------------------------------------------ */
/* Lanczos + ground state                                             */
/* ------------------------------------------------------------------ */

static zc dotc(int64_t n, const zc *a, const zc *b)
{
    zc z = 0;
    for (int64_t i = 0; i < n; i++) z = z + conj(a[i]) * b[i];
    return z;
}

static double norm2(int64_t n, const zc *a)
{
    double m = 0;
    for (int64_t i = 0; i < n; i++) m = m + creal(a[i]) * creal(a[i]) + cimag(a[i]) * cimag(a[i]);
    return sqrt(m);
}

/* Lanczos with one classical Gram-Schmidt reorthogonalisation per step
 * (groundStateLieb.c:217-344). lvec holds lm vectors of nc (lvec[0] = start).
 * diag/offdiag as in the reference (complex, offdiag real-valued). Returns
 * the number of iterations completed (lm unless it broke down). H.psi is
 * orc_apply_h in the given mode (maps optional). */
int orc_lanczos(int N, int M, int mode, const int32_t *IF, const int32_t *Map,
                const int32_t *MapOT, const int64_t *sOT, const int32_t *MapTT,
                const int64_t *sTT, const zc *Ho, const zc *Hint, int lm, zc *lvec,
                zc *diag, zc *offdiag, int nthreads)
{
    int64_t nc = orc_nc(N, M);
    double maxCheck = 0, tol = 1e-15;
    zc *HC = (zc *)malloc(sizeof(zc) * nc);
    zc *ortho = (zc *)malloc(sizeof(zc) * lm);
    if (!HC || !ortho) { free(HC); free(ortho); return -1; }
#define V(k) (lvec + (int64_t)(k) * nc)
    orc_apply_h(N, M, mode, IF, Map, MapOT, sOT, MapTT, sTT, V(0), Ho, Hint, HC, 0, nc, nthreads);
    diag[0] = dotc(nc, V(0), HC);
    for (int64_t j = 0; j < nc; j++) HC[j] = HC[j] - diag[0] * V(0)[j];
    for (int i = 0; i < lm - 1; i++) {
        offdiag[i] = norm2(nc, HC);
        if (maxCheck < creal(offdiag[i])) maxCheck = creal(offdiag[i]);
        if (creal(offdiag[i]) / maxCheck < tol) { free(HC); free(ortho); return i; }
        for (int64_t j = 0; j < nc; j++) V(i + 1)[j] = HC[j] / offdiag[i];
        orc_apply_h(N, M, mode, IF, Map, MapOT, sOT, MapTT, sTT, V(i + 1), Ho, Hint, HC, 0, nc,
                    nthreads);
        for (int64_t j = 0; j < nc; j++) HC[j] = HC[j] - offdiag[i] * V(i)[j];
        diag[i + 1] = dotc(nc, V(i + 1), HC);
        for (int64_t j = 0; j < nc; j++) HC[j] = HC[j] - diag[i + 1] * V(i + 1)[j];
        for (int j = 0; j < i + 2; j++) ortho[j] = dotc(nc, V(j), HC);
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int64_t j = 0; j < nc; j++) {
            zc u = HC[j];
            for (int k = 0; k < i + 2; k++) u = u - V(k)[j] * ortho[k];
            HC[j] = u;
        }
    }
#undef V
    free(HC);
    free(ortho);
    return lm;
}

/* Lowest eigenpair from Niter Lanczos steps started at C
 * (groundStateLieb.c:348-471); C is overwritten with the Ritz vector.
 * Returns the eigenvalue; *iters gets the number of steps done. */
double orc_ground(int N, int M, int mode, const int32_t *IF, const int32_t *Map,
                  const int32_t *MapOT, const int64_t *sOT, const int32_t *MapTT,
                  const int64_t *sTT, const zc *Ho, const zc *Hint, int Niter, zc *C,
                  int *iters, int nthreads)
{
    int64_t nc = orc_nc(N, M);
    double *d = (double *)malloc(sizeof(double) * Niter);
    double *e = (double *)malloc(sizeof(double) * Niter);
    double *ev = (double *)malloc(sizeof(double) * Niter * Niter);
    zc *diag = (zc *)malloc(sizeof(zc) * Niter);
    zc *offdiag = (zc *)malloc(sizeof(zc) * Niter);
    zc *lvec = (zc *)malloc(sizeof(zc) * Niter * nc);
    if (!d || !e || !ev || !diag || !offdiag || !lvec) return NAN;
    offdiag[Niter - 1] = 0;
    for (int64_t i = 0; i < nc; i++) lvec[i] = C[i];
    int it = orc_lanczos(N, M, mode, IF, Map, MapOT, sOT, MapTT, sTT, Ho, Hint, Niter, lvec, diag,
                         offdiag, nthreads);
    if (iters) *iters = it;
    for (int k = 0; k < it; k++) {
        d[k] = creal(diag[k]);
        e[k] = creal(offdiag[k]);
    }
    LAPACKE_dstev(LAPACK_ROW_MAJOR, 'V', it, d, e, ev, it);
    double sentinel = 1e10;
    int jmin = 0;
    for (int k = 0; k < it; k++)
        if (sentinel > d[k]) { sentinel = d[k]; jmin = k; }
    for (int64_t i = 0; i < nc; i++) {
        C[i] = 0;
        for (int k = 0; k < it; k++) C[i] += lvec[(int64_t)k * nc + i] * ev[k * it + jmin];
    }
    free(d); free(e); free(ev); free(diag); free(offdiag); free(lvec);
    return sentinel;
}
