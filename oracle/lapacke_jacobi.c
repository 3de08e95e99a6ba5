/* Oracle-side LAPACKE_dstev (test infrastructure only).
 *
 * The reference's ground-state driver diagonalises the real symmetric
 * tridiagonal Lanczos matrix with MKL's LAPACKE_dstev('V')
 * (groundStateLieb.c:428-440): eigenvalues ascending in d, eigenvectors in z
 * (row-major: z[k*ldz + j] is component k of eigenvector j). MKL is absent
 * here, so the oracle supplies its own routine with that contract: the
 * tridiagonal is expanded to a dense matrix and diagonalised by the cyclic
 * Jacobi method (Jacobi 1846; rotation formulas as in Rutishauser's 1966
 * "The Jacobi method for real symmetric matrices"), then sorted ascending.
 * Jacobi is slower than QL but has high relative accuracy and shares no code
 * with the product's implicit-QL solver, so the two cross-check each other. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "mkl.h"

static void jacobi_sym(int n, double *a, double *v)
{
    for (int i = 0; i < n * n; i++) v[i] = 0.0;
    for (int i = 0; i < n; i++) v[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int p = 0; p < n; p++) {
            diag += a[p * n + p] * a[p * n + p];
            for (int q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
        }
        if (off <= 1e-34 * (diag + 1e-300)) break;
        for (int p = 0; p < n; p++) {
            for (int q = p + 1; q < n; q++) {
                double apq = a[p * n + q];
                if (apq == 0.0) continue;
                double app = a[p * n + p], aqq = a[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) /
                           (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) {       /* columns p,q */
                    double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = c * akp - s * akq;
                    a[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {       /* rows p,q */
                    double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = c * apk - s * aqk;
                    a[q * n + k] = s * apk + c * aqk;
                }
                a[p * n + q] = a[q * n + p] = 0.0;
                for (int k = 0; k < n; k++) {       /* accumulate V */
                    double vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = c * vkp - s * vkq;
                    v[k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
}

lapack_int LAPACKE_dstev(int layout, char jobz, lapack_int n, double *d,
                         double *e, double *z, lapack_int ldz)
{
    if (n < 0) return -3;
    if (n == 0) return 0;
    double *a = (double *)calloc((size_t)n * n, sizeof(double));
    double *v = (double *)malloc((size_t)n * n * sizeof(double));
    int *perm = (int *)malloc((size_t)n * sizeof(int));
    if (!a || !v || !perm) { free(a); free(v); free(perm); return -1010; }
    for (int i = 0; i < n; i++) {
        a[i * n + i] = d[i];
        if (i + 1 < n) a[i * n + i + 1] = a[(i + 1) * n + i] = e[i];
    }
    jacobi_sym(n, a, v);
    for (int i = 0; i < n; i++) perm[i] = i;
    for (int i = 1; i < n; i++) {              /* insertion sort, ascending */
        int pi = perm[i], j = i - 1;
        while (j >= 0 && a[perm[j] * n + perm[j]] > a[pi * n + pi]) {
            perm[j + 1] = perm[j];
            j--;
        }
        perm[j + 1] = pi;
    }
    for (int j = 0; j < n; j++) d[j] = a[perm[j] * n + perm[j]];
    if (jobz == 'V' || jobz == 'v') {
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++) {
                double val = v[k * n + perm[j]];
                if (layout == LAPACK_ROW_MAJOR) z[(size_t)k * ldz + j] = val;
                else z[k + (size_t)j * ldz] = val;
            }
    }
    free(a); free(v); free(perm);
    return 0;
}
