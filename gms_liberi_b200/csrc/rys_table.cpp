// rys_table.cpp -- piecewise-polynomial Rys roots and weights for 1..5 roots
// (s/p/d classes) and 1..7 roots (f classes).
//
// The reference computes Rys roots per primitive quartet by a 35-point
// discretised Stieltjes procedure followed by Golub-Welsch
// (src/rhf/rot_axis/int2222_rysgen.F90:636-877), and Boys-table interpolation
// in the rotated-axis kernels (src/liberi_boys.F90).  On the GPU that per-
// quartet work is replaced by tables built here once per process:
//   * exact roots u_i(T) = t_i^2 and weights w_i(T) of the Rys weight
//     exp(-T t^2) on [0,1] are computed at Chebyshev nodes of every interval
//     [k/4, (k+1)/4), k = 0..239, from the recurrence coefficients of a
//     64-point Gauss-Legendre discretisation (Stieltjes procedure) and Sturm
//     bisection of the Jacobi matrix, weights by Christoffel numbers;
//   * each root and weight is interpolated by a degree-7 Chebyshev
//     polynomial per interval and stored in power form of x = 2(4T-k)-1
//     (8 coefficients), which the device evaluates with Estrin's scheme
//     (7 FMAs, dependency depth 3) from 4 aligned double2 loads.
// Interpolation error is below 6e-15 relative (checked by the unit tests
// against the oracle's 35-point procedure).  Above the class threshold the device
// uses the large-T (Gauss-Hermite) limit, built here as well.  A second,
// single-precision set (intervals of width 1/8, degree 3) serves the FP32
// tier of the mixed-precision build.  The f classes' table covers 1..7 roots
// on [0, 65) in the same form (the reference's 6- and 7-root kernels switch
// to the large-T limit at 60 and 65, int3322_rysgen.F90, int3333_rysgen.F90:1206).
#include <cmath>
#include <mutex>
#include <vector>

#include "engine.h"

namespace liberi {
namespace {

const double PI = 3.14159265358979323846;

void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.resize(n);
    w.resize(n);
    for (int i = 0; i < n; i++) {
        double z = std::cos(PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            dp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / dp;
            if (std::fabs(z - z1) < 1e-16) break;
        }
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// Gauss rule of a Jacobi matrix: diag a[0..n-1], squared off-diagonals
// b2[1..n-1], total mass beta0; nodes in [lo, hi] ascending.
void jacobi_rule(int n, const double *a, const double *b2, double beta0, double lo, double hi,
                 double *x, double *w) {
    auto count_below = [&](double s) {
        int c = 0;
        double q = a[0] - s;
        if (q < 0) c++;
        for (int i = 1; i < n; i++) {
            if (q == 0.0) q = 1e-300;
            q = a[i] - s - b2[i] / q;
            if (q < 0) c++;
        }
        return c;
    };
    for (int k = 0; k < n; k++) {
        double l = lo, h = hi;
        for (int it = 0; it < 200; it++) {
            double m = 0.5 * (l + h);
            if (m <= l || m >= h) break;
            if (count_below(m) > k) h = m; else l = m;
        }
        double r = 0.5 * (l + h);
        double p0 = 1.0, p1 = 0.0, norm = 1.0, s = 1.0;
        for (int j = 0; j + 1 < n; j++) {
            double pn = (r - a[j]) * p0 - (j > 0 ? b2[j] * p1 : 0.0);
            p1 = p0;
            p0 = pn;
            norm *= b2[j + 1];
            s += p0 * p0 / norm;
        }
        x[k] = r;
        w[k] = beta0 / s;
    }
}

struct Grid {
    std::vector<double> u, w;
    Grid() {
        std::vector<double> x, wx;
        gauss_legendre(64, x, wx);
        for (size_t i = 0; i < x.size(); i++) {
            double t = 0.5 * (x[i] + 1.0);
            u.push_back(t * t);
            w.push_back(0.5 * wx[i]);
        }
    }
};

void exact_rys(const Grid &g, int n, double T, double *u, double *w) {
    const int N = (int)g.u.size();
    std::vector<double> W(N), p0(N, 1.0), p1(N, 0.0);
    double s0 = 0, s1 = 0;
    for (int j = 0; j < N; j++) {
        W[j] = g.w[j] * std::exp(-T * g.u[j]);
        s0 += W[j];
        s1 += W[j] * g.u[j];
    }
    double a[MAXROOT7], b2[MAXROOT7];
    a[0] = s1 / s0;
    b2[0] = 0.0;
    double prev = s0;
    for (int k = 1; k < n; k++) {
        double sa = 0, sb = 0;
        for (int j = 0; j < N; j++) {
            double pn = (g.u[j] - a[k - 1]) * p0[j] - (k > 1 ? b2[k - 1] * p1[j] : 0.0);
            p1[j] = p0[j];
            p0[j] = pn;
            sa += W[j] * pn * pn;
            sb += W[j] * g.u[j] * pn * pn;
        }
        a[k] = sb / sa;
        b2[k] = sa / prev;
        prev = sa;
    }
    jacobi_rule(n, a, b2, s0, 0.0, 1.0, u, w);
}

std::vector<double> g_table;
std::once_flag g_once;
std::vector<float> g_table_f;
std::once_flag g_once_f;

// Chebyshev interpolation of f at the M nodes of [-1, 1], converted to the
// power basis of x (coefficients 0..M-1).
std::vector<double> cheb_to_power(const std::vector<double> &f) {
    const int M = (int)f.size();
    std::vector<double> c(M, 0.0);
    for (int j = 0; j < M; j++) {
        double s = 0.0;
        for (int m = 0; m < M; m++) s += f[m] * std::cos(PI * j * (m + 0.5) / M);
        c[j] = 2.0 * s / M;
    }
    c[0] *= 0.5;
    std::vector<double> pw(M, 0.0), tprev(M, 0.0), tcur(M, 0.0);
    tcur[0] = 1.0;
    for (int j = 0; j < M; j++) {
        if (j == 1) {
            tprev = tcur;
            std::fill(tcur.begin(), tcur.end(), 0.0);
            tcur[1] = 1.0;
        } else if (j > 1) {
            std::vector<double> tn(M, 0.0);
            for (int i = 0; i + 1 < M; i++) tn[i + 1] += 2.0 * tcur[i];
            for (int i = 0; i < M; i++) tn[i] -= tprev[i];
            tprev = tcur;
            tcur = tn;
        }
        for (int i = 0; i < M; i++) pw[i] += c[j] * tcur[i];
    }
    return pw;
}

// FP32 tier: width-1/8 intervals, degree 3: one float4 per function, the
// power-basis coefficients small, single-precision evaluation within a few
// float ulps of the exact roots and weights.
void build_tables_f32() {
    Grid g;
    const std::vector<double> &dt = rys_table_host();
    g_table_f.assign(RYSF_TABLE_SIZE, 0.0f);
    const int M = RYSF_DEG + 1;
    std::vector<double> xs(M);
    for (int m = 0; m < M; m++) xs[m] = std::cos(PI * (m + 0.5) / M);
    for (int n = 1; n <= MAXROOT; n++) {
        for (int k = 0; k < RYSF_NINT; k++) {
            std::vector<std::vector<double>> f(2 * n, std::vector<double>(M));
            for (int m = 0; m < M; m++) {
                double T = (k + 0.5 * (xs[m] + 1.0)) / RYSF_PER_UNIT;
                double u[MAXROOT], w[MAXROOT];
                exact_rys(g, n, T, u, w);
                for (int i = 0; i < n; i++) {
                    f[i][m] = u[i];
                    f[n + i][m] = w[i];
                }
            }
            for (int fi = 0; fi < 2 * n; fi++) {
                std::vector<double> pw = cheb_to_power(f[fi]);
                float *dst = &g_table_f[rysf_table_off(n) + ((size_t)k * 2 * n + fi) * RYSF_NCOEF];
                for (int i = 0; i < M; i++) dst[i] = (float)pw[i];
            }
        }
        for (int i = 0; i < 2 * MAXROOT; i++) g_table_f[rysf_herm_off(n) + i] = (float)dt[rys_herm_off(n) + i];
    }
}

// Double-precision table of 1..nmax roots over nint intervals of width
// 1/RYS_PER_UNIT: per n and interval, 2n functions (roots, then weights) of
// RYS_NCOEF power-basis coefficients at tab_off(n); then per n the large-T
// limit (nmax Gauss-Hermite r_i, then nmax W_i) at herm_off(n).
template <typename OffT, typename HermT>
void fill_table(int nmax, int nint, OffT tab_off, HermT herm_off, std::vector<double> &out) {
    Grid g;
    const int M = RYS_DEG + 1;  // interpolation nodes / coefficients
    std::vector<double> xs(M);
    for (int m = 0; m < M; m++) xs[m] = std::cos(PI * (m + 0.5) / M);
    for (int n = 1; n <= nmax; n++) {
        for (int k = 0; k < nint; k++) {
            std::vector<std::vector<double>> f(2 * n, std::vector<double>(M));
            for (int m = 0; m < M; m++) {
                double T = (k + 0.5 * (xs[m] + 1.0)) / RYS_PER_UNIT;
                double u[MAXROOT7], w[MAXROOT7];
                exact_rys(g, n, T, u, w);
                for (int i = 0; i < n; i++) {
                    f[i][m] = u[i];
                    f[n + i][m] = w[i];
                }
            }
            for (int fi = 0; fi < 2 * n; fi++) {
                std::vector<double> pw = cheb_to_power(f[fi]);
                double *dst = &out[tab_off(n) + ((size_t)k * 2 * n + fi) * RYS_NCOEF];
                for (int i = 0; i < M; i++) dst[i] = pw[i];
                for (int i = M; i < RYS_NCOEF; i++) dst[i] = 0.0;
            }
        }
    }
    // Gauss-Hermite (2n points) positive half: large-T limit
    for (int n = 1; n <= nmax; n++) {
        int m = 2 * n;
        double a[2 * MAXROOT7], b2[2 * MAXROOT7], x[2 * MAXROOT7], w[2 * MAXROOT7];
        for (int i = 0; i < m; i++) {
            a[i] = 0.0;
            b2[i] = 0.5 * i;
        }
        jacobi_rule(m, a, b2, std::sqrt(PI), -(double)m, (double)m, x, w);
        for (int i = 0; i < n; i++) {
            out[herm_off(n) + i] = x[n + i] * x[n + i];
            out[herm_off(n) + nmax + i] = w[n + i];
        }
    }
}

void build_tables() {
    g_table.assign(RYS_TABLE_SIZE, 0.0);
    fill_table(MAXROOT, RYS_NINT, rys_table_off, rys_herm_off, g_table);
}

std::vector<double> g_table7;
std::once_flag g_once7;

void build_tables7() {
    g_table7.assign(RYS7_TABLE_SIZE, 0.0);
    fill_table(MAXROOT7, RYS7_NINT, rys7_table_off, rys7_herm_off, g_table7);
}

}  // namespace

const std::vector<double> &rys_table_host() {
    std::call_once(g_once, build_tables);
    return g_table;
}

const std::vector<float> &rys_table_f32_host() {
    std::call_once(g_once_f, build_tables_f32);
    return g_table_f;
}

const std::vector<double> &rys_table7_host() {
    std::call_once(g_once7, build_tables7);
    return g_table7;
}


}  // namespace liberi
