// small_linalg.cuh -- dense M x M complex128 kernels (M <= 30) used by the
// density-matrix synchronisation (synchronize.c:42-57 of the reference,
// which calls LAPACK zheev / zhesv through lapack_interface.c:61-163):
//   * Hermitian eigen-decomposition by cyclic Jacobi rotations,
//   * Hermitian inverse by Gauss-Jordan elimination with partial pivoting,
//   * the regularisation A += x exp(-A / x) (lapack_interface.c:126);
// and the real symmetric tridiagonal eigenproblem of the Lanczos step (in
// place of LAPACK dstev, multiconfig_lanczos.c:143).
// Row-major double2 storage; usable from host code and from one device
// thread.  Results agree with LAPACK to rounding for the well-conditioned
// one-body density matrices these are applied to.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace mctdhb {

__host__ __device__ inline double2 c_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ inline double c_abs(double2 a) { return hypot(a.x, a.y); }

// Eigenvalues ascending in w[n]; eigenvectors in the columns of v (row-major,
// may be null).  `a` is overwritten.  Returns the sweeps used (<= 100).
__host__ __device__ inline int herm_eig_jacobi(int n, double2* a, double* w, double2* v) {
    if (v)
        for (int i = 0; i < n * n; i++) v[i] = make_double2((i / n == i % n) ? 1.0 : 0.0, 0.0);
    int sweep = 0;
    for (; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int p = 0; p < n; p++)
            for (int q = 0; q < n; q++) {
                const double m2 = a[p * n + q].x * a[p * n + q].x + a[p * n + q].y * a[p * n + q].y;
                tot += m2;
                if (p != q) off += m2;
            }
        if (off == 0.0 || off <= 1e-30 * tot) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double2 apq = a[p * n + q];
                const double mag = c_abs(apq);
                if (mag == 0.0) continue;
                const double2 ph = make_double2(apq.x / mag, apq.y / mag);
                const double theta = 0.5 * atan2(2.0 * mag, a[q * n + q].x - a[p * n + p].x);
                const double c = cos(theta), s = sin(theta);
                // A <- J^H A J, J = [[c, s ph], [-s conj(ph), c]] in the (p, q) plane
                for (int k = 0; k < n; k++) {
                    const double2 akp = a[k * n + p], akq = a[k * n + q];
                    const double2 t1 = c_mul(c_conj(ph), akq), t2 = c_mul(ph, akp);
                    a[k * n + p] = make_double2(c * akp.x - s * t1.x, c * akp.y - s * t1.y);
                    a[k * n + q] = make_double2(s * t2.x + c * akq.x, s * t2.y + c * akq.y);
                }
                for (int k = 0; k < n; k++) {
                    const double2 apk = a[p * n + k], aqk = a[q * n + k];
                    const double2 t1 = c_mul(ph, aqk), t2 = c_mul(c_conj(ph), apk);
                    a[p * n + k] = make_double2(c * apk.x - s * t1.x, c * apk.y - s * t1.y);
                    a[q * n + k] = make_double2(s * t2.x + c * aqk.x, s * t2.y + c * aqk.y);
                }
                if (v)
                    for (int k = 0; k < n; k++) {
                        const double2 vkp = v[k * n + p], vkq = v[k * n + q];
                        const double2 t1 = c_mul(c_conj(ph), vkq), t2 = c_mul(ph, vkp);
                        v[k * n + p] = make_double2(c * vkp.x - s * t1.x, c * vkp.y - s * t1.y);
                        v[k * n + q] = make_double2(s * t2.x + c * vkq.x, s * t2.y + c * vkq.y);
                    }
            }
    }
    // selection sort ascending, permuting eigenvector columns
    for (int i = 0; i < n; i++) w[i] = a[i * n + i].x;
    for (int i = 0; i < n; i++) {
        int best = i;
        for (int j = i + 1; j < n; j++)
            if (w[j] < w[best]) best = j;
        if (best != i) {
            const double t = w[i];
            w[i] = w[best];
            w[best] = t;
            if (v)
                for (int k = 0; k < n; k++) {
                    const double2 u = v[k * n + i];
                    v[k * n + i] = v[k * n + best];
                    v[k * n + best] = u;
                }
        }
    }
    return sweep;
}

// inv = A^{-1}; `a` is overwritten.  Returns 0, or k+1 when column k has no
// non-zero pivot (singular).
__host__ __device__ inline int herm_inverse(int n, double2* a, double2* inv) {
    for (int i = 0; i < n * n; i++) inv[i] = make_double2((i / n == i % n) ? 1.0 : 0.0, 0.0);
    for (int c = 0; c < n; c++) {
        int piv = c;
        double best = c_abs(a[c * n + c]);
        for (int r = c + 1; r < n; r++) {
            const double v = c_abs(a[r * n + c]);
            if (v > best) {
                best = v;
                piv = r;
            }
        }
        if (best == 0.0) return c + 1;
        if (piv != c)
            for (int k = 0; k < n; k++) {
                double2 t = a[c * n + k];
                a[c * n + k] = a[piv * n + k];
                a[piv * n + k] = t;
                t = inv[c * n + k];
                inv[c * n + k] = inv[piv * n + k];
                inv[piv * n + k] = t;
            }
        const double2 d = a[c * n + c];
        const double dd = d.x * d.x + d.y * d.y;
        const double2 r = make_double2(d.x / dd, -d.y / dd);
        for (int k = 0; k < n; k++) {
            a[c * n + k] = c_mul(a[c * n + k], r);
            inv[c * n + k] = c_mul(inv[c * n + k], r);
        }
        for (int row = 0; row < n; row++) {
            if (row == c) continue;
            const double2 f = a[row * n + c];
            if (f.x == 0.0 && f.y == 0.0) continue;
            for (int k = 0; k < n; k++) {
                const double2 t1 = c_mul(f, a[c * n + k]), t2 = c_mul(f, inv[c * n + k]);
                a[row * n + k].x -= t1.x;
                a[row * n + k].y -= t1.y;
                inv[row * n + k].x -= t2.x;
                inv[row * n + k].y -= t2.y;
            }
        }
    }
    return 0;
}

// rho1 <- regularised rho1 and rinv = rho1^{-1} following synchronize.c:42-57:
// if lambda_min / lambda_max < reg_fac, add x exp(-rho1 / x) with
// x = lambda_max reg_fac (lapack_interface.c:126-163).  `work` holds 3 n^2
// double2 and n doubles.  Returns 0, or the inverse's error code.
__host__ __device__ inline int sync_rho1(int n, double2* rho1, double2* rinv, double reg_fac,
                                         double2* work, double* wd) {
    double2* a = work;
    double2* v = work + n * n;
    for (int i = 0; i < n * n; i++) a[i] = rho1[i];
    herm_eig_jacobi(n, a, wd, v);
    if (wd[0] / wd[n - 1] < reg_fac) {
        const double x = wd[n - 1] * reg_fac;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double2 z = make_double2(0.0, 0.0);
                for (int k = 0; k < n; k++) {
                    const double f = x * exp(-wd[k] / x);
                    const double2 t = c_mul(v[i * n + k], c_conj(v[j * n + k]));
                    z.x += f * t.x;
                    z.y += f * t.y;
                }
                rho1[i * n + j].x += z.x;
                rho1[i * n + j].y += z.y;
            }
    }
    for (int i = 0; i < n * n; i++) a[i] = rho1[i];
    return herm_inverse(n, a, rinv);
}

// Implicit QL with Wilkinson shifts for the symmetric tridiagonal matrix
// (d, e); eigenvectors accumulate in the columns of row-major z (n x n).
__host__ __device__ inline int tridiag_ql(int n, double* d, double* e, double* z) {
    for (int i = 0; i < n * n; i++) z[i] = 0.0;
    for (int i = 0; i < n; i++) z[i * n + i] = 1.0;
    if (n < 1) return 0;
    e[n - 1] = 0.0;
    for (int l = 0; l < n; l++) {
        int iter = 0;
        for (;;) {
            int m;
            for (m = l; m < n - 1; m++) {
                const double dd = fabs(d[m]) + fabs(d[m + 1]);
                if (fabs(e[m]) <= 2.220446049250313e-16 * dd) break;
            }
            if (m == l) break;
            if (++iter > 60) return l + 1;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? fabs(r) : -fabs(r)));
            double s = 1.0, c = 1.0, p = 0.0;
            bool deflated = false;
            for (int i = m - 1; i >= l; i--) {
                double f = s * e[i];
                const double b = c * e[i];
                r = hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
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
                for (int k = 0; k < n; k++) {
                    f = z[k * n + i + 1];
                    z[k * n + i + 1] = s * z[k * n + i] + c * f;
                    z[k * n + i] = c * z[k * n + i] - s * f;
                }
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

}  // namespace mctdhb
