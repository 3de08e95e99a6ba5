// Symmetric tridiagonal eigensolver for the Lanczos matrix.
//
// The reference diagonalises the Lanczos tridiagonal with MKL's
// LAPACKE_dstev('V') (groundStateLieb.c:428-440). This is an own
// implementation of the implicit QL algorithm with Wilkinson shifts
// (Bowdler, Martin, Reinsch & Wilkinson, Numer. Math. 11 (1968) 293-306),
// accumulating the plane rotations into the eigenvector matrix, followed by an
// ascending sort. Contract as LAPACKE_dstev(ROW_MAJOR, 'V'): on return d holds
// the eigenvalues ascending and z[k*n + j] is component k of eigenvector j.
#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <vector>

namespace mcpi {

int tridiag_eig(int n, double *d, const double *e_in, double *z)
{
    if (n <= 0) return 0;
    std::vector<double> e(n, 0.0);
    for (int i = 0; i + 1 < n; ++i) e[i] = e_in[i];
    std::vector<double> Z;
    if (z) {
        Z.assign((size_t)n * n, 0.0);
        for (int i = 0; i < n; ++i) Z[(size_t)i * n + i] = 1.0;
    }
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        for (;;) {
            int m = l;
            for (; m < n - 1; ++m) {
                const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= eps * dd) break;
            }
            if (m == l) break;
            if (++iter > 64) return -1;
            // Wilkinson-type shift from the leading 2x2 block
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = m - 1;
            bool deflated = false;
            for (; i >= l; --i) {
                const double f = s * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {  // underflow: split the matrix here
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                if (z) {
                    for (int k = 0; k < n; ++k) {
                        double *zk = &Z[(size_t)k * n];
                        const double fz = zk[i + 1];
                        zk[i + 1] = s * zk[i] + c * fz;
                        zk[i] = c * zk[i] - s * fz;
                    }
                }
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return d[a] < d[b]; });
    std::vector<double> ds(d, d + n);
    for (int j = 0; j < n; ++j) d[j] = ds[perm[j]];
    if (z)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j) z[(size_t)k * n + j] = Z[(size_t)k * n + perm[j]];
    return 0;
}

}  // namespace mcpi
