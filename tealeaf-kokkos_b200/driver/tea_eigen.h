// Host-side FP64 scalar algorithms of the Chebyshev/PPCG switch, shared by the driver
// (per-call path) and by the CUDA library's whole-solve entry point, so both compute
// identical eigenvalue estimates, coefficients and iteration estimates.
//
//   tea_tqli              tealeaf_2d/tea_leaf_cheby.f90:233-283 (QL with implicit shifts
//                         on a symmetric tridiagonal matrix, as restated from the reference)
//   tea_calc_eigenvalues  tealeaf_2d/tea_leaf_cheby.f90:285-332 (Lanczos tridiagonal built
//                         from the CG alphas/betas, then sorted)
//   tea_calc_ch_coefs     tealeaf_2d/tea_leaf_cheby.f90:334-360 (Chebyshev recurrence)
//   tea_cheby_est_itc     tealeaf_2d/tea_solve.f90:739-741
//
// All arrays are 0-based here; the Fortran is 1-based.  Host code including this file
// must be compiled with FP contraction off (-ffp-contract=off), as the library is.
#ifndef TEA_EIGEN_H
#define TEA_EIGEN_H

#include <cmath>
#include <vector>

namespace tea {

// The reference scales the eigenvalue bounds by the default-real (single precision)
// literals 0.95 and 1.05 (tealeaf_2d/tea_solve.f90:194-195).
constexpr double kEigMinScale = (double)0.95f;
constexpr double kEigMaxScale = (double)1.05f;

// Returns 0 on success, 1 when an eigenvalue did not converge in 30 sweeps.
inline int tea_tqli(std::vector<double>& d, std::vector<double>& e)
{
    const int n = (int)d.size();
    // e(:) = eoshift(e(:), 1)
    for (int i = 0; i + 1 < n; ++i) e[i] = e[i + 1];
    if (n > 0) e[n - 1] = 0.0;
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        for (;;) {
            int m;
            for (m = l; m < n - 1; ++m) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) + dd == dd) break;
            }
            if (m == l) break;
            if (iter == 30) return 1;
            ++iter;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::sqrt(g * g + 1.0);
            g = d[m] - d[l] + e[l] / (g + std::copysign(std::fabs(r), g));
            double s = 1.0, c = 1.0, p = 0.0;
            bool restart = false;
            for (int i = m - 1; i >= l; --i) {
                double f = s * e[i];
                double b = c * e[i];
                r = std::sqrt(f * f + g * g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] = d[i + 1] - p;
                    e[m] = 0.0;
                    restart = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
            }
            if (restart) continue;
            d[l] = d[l] - p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

// cg_alphas/cg_betas hold the first `n` CG scalars (n = switch step - 1).
// Returns info: 0 ok, 1 failure (tqli) or a negative bound.
inline int tea_calc_eigenvalues(const double* cg_alphas, const double* cg_betas, int n,
                                double* eigmin, double* eigmax)
{
    if (n < 1) return 1;
    std::vector<double> diag(n, 0.0), offdiag(n, 0.0);
    for (int k = 0; k < n; ++k) {
        diag[k] = 1.0 / cg_alphas[k];
        if (k > 0) diag[k] = diag[k] + cg_betas[k - 1] / cg_alphas[k - 1];
        if (k < n - 1) offdiag[k + 1] = std::sqrt(cg_betas[k]) / cg_alphas[k];
    }
    int info = tea_tqli(diag, offdiag);
    if (info != 0) return info;
    // Bubble sort with the reference's >= test (tealeaf_2d/tea_leaf_cheby.f90:314-325).
    // Equal neighbours would swap forever there; the pass count is bounded here.
    bool swapped = false;
    for (int pass = 0; pass < n + 2; ++pass) {
        for (int k = 0; k + 1 < n; ++k) {
            if (diag[k] >= diag[k + 1]) {
                double tmp = diag[k];
                diag[k] = diag[k + 1];
                diag[k + 1] = tmp;
                swapped = true;
            }
        }
        if (!swapped) break;
        swapped = false;
    }
    *eigmin = diag[0];
    *eigmax = diag[n - 1];
    if (*eigmin < 0.0 || *eigmax < 0.0) info = 1;
    return info;
}

inline void tea_calc_ch_coefs(double* ch_alphas, double* ch_betas, double eigmin, double eigmax,
                              double* theta, int n)
{
    *theta = (eigmax + eigmin) / 2.0;
    const double delta = (eigmax - eigmin) / 2.0;
    const double sigma = *theta / delta;
    double rho_old = 1.0 / sigma;
    for (int k = 0; k < n; ++k) {
        const double rho_new = 1.0 / (2.0 * sigma - rho_old);
        ch_alphas[k] = rho_new * rho_old;
        ch_betas[k] = 2.0 * rho_new / delta;
        rho_old = rho_new;
    }
}

// Smallest and largest eigenvalue of the same Lanczos tridiagonal as tea_calc_eigenvalues
// (from the first `n` CG alphas/betas) by Sturm-sequence bisection: O(n) per step instead
// of the O(n^2) QL sweep, for estimates refreshed while CG runs (the FP32-refined form).
// Not part of the reference's algorithm.  Returns 0 on success, 1 for n < 1.
inline int tea_tridiag_extremes(const double* cg_alphas, const double* cg_betas, int n, double* eigmin,
                                double* eigmax)
{
    if (n < 1) return 1;
    std::vector<double> diag(n), off2(n, 0.0);  // off2[k] = offdiag(k)^2, coupling k-1 and k
    double lo = 0.0, hi = 0.0;
    for (int k = 0; k < n; ++k) {
        diag[k] = 1.0 / cg_alphas[k];
        if (k > 0) diag[k] = diag[k] + cg_betas[k - 1] / cg_alphas[k - 1];
        if (k > 0) off2[k] = cg_betas[k - 1] / (cg_alphas[k - 1] * cg_alphas[k - 1]);
    }
    // Gershgorin interval.
    for (int k = 0; k < n; ++k) {
        const double r = (k > 0 ? std::sqrt(off2[k]) : 0.0) + (k + 1 < n ? std::sqrt(off2[k + 1]) : 0.0);
        lo = k == 0 ? diag[k] - r : std::fmin(lo, diag[k] - r);
        hi = k == 0 ? diag[k] + r : std::fmax(hi, diag[k] + r);
    }
    // Number of eigenvalues below x (Sturm count of the LDL^T pivots).
    auto below = [&](double x) {
        int count = 0;
        double q = 1.0;
        for (int k = 0; k < n; ++k) {
            q = diag[k] - x - (k > 0 ? off2[k] / q : 0.0);
            if (q == 0.0) q = -1e-300;
            if (q < 0.0) ++count;
        }
        return count;
    };
    auto bisect = [&](int index) {  // the eigenvalue with `index` eigenvalues below it
        double a = lo, b = hi;
        for (int it = 0; it < 200 && b - a > 1e-13 * std::fmax(std::fabs(a), std::fabs(b)); ++it) {
            const double m = 0.5 * (a + b);
            if (below(m) > index) b = m;
            else a = m;
        }
        return 0.5 * (a + b);
    };
    *eigmin = bisect(0);
    *eigmax = bisect(n - 1);
    return 0;
}

// NINT(LOG(it_alpha)/(2*LOG(gamm))) with it_alpha = EPSILON(1d0)*bb/(4*error).
inline int tea_cheby_est_itc(double bb, double error, double cn)
{
    const double it_alpha = 2.220446049250313e-16 * bb / (4.0 * error);
    const double gamm = (std::sqrt(cn) - 1.0) / (std::sqrt(cn) + 1.0);
    return (int)std::lround(std::log(it_alpha) / (2.0 * std::log(gamm)));
}

}  // namespace tea

#endif  // TEA_EIGEN_H
