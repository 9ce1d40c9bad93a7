// Kaiser-Bessel splitting on the host (src/BiotSavart/splitting/kaiser_bessel.jl:130-163,
// splitting/chebyshev.jl:12-172).
//
// The reference evaluates the short-range weights 1 - F(r) and r f(r) through Chebyshev series
// of the Kaiser-Bessel kernel f and of its integral F, truncated at the splitting's rtol.  Those
// truncated series define the weights, so they are rebuilt here with the reference's rules and
// then fitted, interval by interval, into the same piecewise-polynomial table layout the pair
// kernels read for the Gaussian weights:
//   table 0: a(x) = 1 - F(r),          table 1: g(x) = 1 - F(r) + r f(r),     x = s r,
// with s = xmax / rcut.  Each interval [c - 1/32, c + 1/32] is interpolated at 10 Chebyshev
// points and the interpolant rewritten in powers of (x - c), so the device evaluates it with the
// same Horner loop as the Gaussian tables.  Fitting values (rather than differentiating the
// series) keeps the tables within a few ulps of the series even when the series carries
// rounding noise at high degree (beta > ~35, where rtol is below the FP64 epsilon).
#include <cmath>
#include <vector>

#include "vpbs_internal.cuh"

namespace vpbs {
namespace {

// Clenshaw evaluation of sum_k c_k T_k(u).
double cheb_eval(const std::vector<double>& c, double u) {
    if (c.empty()) return 0.0;
    double b1 = 0.0, b2 = 0.0;
    for (int k = (int)c.size() - 1; k >= 1; --k) {
        const double b = 2.0 * u * b1 + c[k] - b2;
        b2 = b1;
        b1 = b;
    }
    return c[0] + u * b1 - b2;
}

double kb_kernel(double beta, double rcut, double r) {
    const double u = r / rcut;
    const double s = 1.0 - u * u;
    return beta / (rcut * std::sinh(beta)) * std::cyl_bessel_i(0.0, beta * std::sqrt(s > 0.0 ? s : 0.0));
}

}  // namespace

// chebyshev.jl:130-172 (approximate with symmetry = :even) and 73-122 (integrate): the
// Chebyshev coefficients of f on the N-point extrema grid r_n = rcut cos(pi n / (N - 1)) (a
// type-I cosine transform, ends halved, divided by N - 1), cut before the first two
// consecutive coefficients below rtol * sum |c| (N doubling from 64 until such a pair
// exists), odd coefficients dropped; then the term-by-term integral, scaled by rcut.  Both
// series are returned as full coefficient vectors in u = r / rcut.
KBSeries kb_series(double beta, double rcut, double rtol) {
    KBSeries S;
    S.beta = beta;
    S.rcut = rcut;
    std::vector<double> cs;
    int cut = -1;
    for (int N = 64; N <= 4096; N *= 2) {
        std::vector<double> us(N);
        for (int n = 0; n < N; ++n) us[n] = kb_kernel(beta, rcut, rcut * std::cos(kPi * n / (N - 1)));
        cs.assign(N, 0.0);
        for (int k = 0; k < N; ++k) {
            double acc = us[0] + ((k % 2) ? -us[N - 1] : us[N - 1]);
            for (int j = 1; j < N - 1; ++j) acc += 2.0 * us[j] * std::cos(kPi * (double)((int64_t)j * k % (2 * (N - 1))) / (N - 1));
            cs[k] = acc;
        }
        cs[0] *= 0.5;
        cs[N - 1] *= 0.5;
        double sum = 0.0;
        for (double& c : cs) {
            c /= (N - 1);
            sum += std::fabs(c);
        }
        const double atol = rtol * sum;
        for (int j = 0; j + 1 < N; ++j)
            if (std::fabs(cs[j]) < atol && std::fabs(cs[j + 1]) < atol) {
                cut = j;
                break;
            }
        if (cut >= 0) break;
    }
    if (cut < 1) return S;  // empty: the caller reports the failure
    std::vector<double> e;
    for (int j = 0; j < cut; j += 2) e.push_back(cs[j]);
    const int n = (int)e.size();
    S.f.assign(2 * n - 1, 0.0);
    for (int i = 0; i < n; ++i) S.f[2 * i] = e[i];
    std::vector<double> o(n);
    if (n == 1) {
        o[0] = e[0];
    } else {
        o[0] = (2.0 * e[0] - e[1]) / 2.0;
        for (int i = 1; i < n - 1; ++i) o[i] = (e[i] - e[i + 1]) / (2.0 * (2 * i + 1));
        o[n - 1] = e[n - 1] / (2.0 * (2 * n - 1));
    }
    S.F.assign(2 * n, 0.0);
    for (int i = 0; i < n; ++i) S.F[2 * i + 1] = o[i] * rcut;
    return S;
}

// a = 1 - F(r) and g = 1 - F(r) + r f(r) from the two series (weights_shortrange,
// kaiser_bessel.jl:282-292: the velocity integrand takes a + b = g, the streamfunction a).
void kb_weights_series(const KBSeries& S, double r, double* a, double* g) {
    const double u = r / S.rcut;
    const double A = 1.0 - cheb_eval(S.F, u);
    *a = A;
    *g = A + r * cheb_eval(S.f, u);
}

double kb_table_xmax(double beta) {
    const double w = std::sqrt(beta / 2.0);
    return 1.5 * (w > 2.0 ? w : 2.0);
}

// Tables in the layout of ewald_table_host: ntab intervals of width 1/16 in x = s r (s = xmax /
// rcut), kEwaldNC coefficients in powers of (x - c) per interval, table a then table g.
void kb_table_host(const KBSeries& S, int* ntab, double* tab) {
    const double xmax = kb_table_xmax(S.beta);
    const int K = ewald_table_size(xmax);
    *ntab = K;
    if (!tab) return;
    const double s = xmax / S.rcut;
    constexpr int n = kEwaldNC;
    const double h = 0.5 * kEwaldH;
    // monomial coefficients of T_0 .. T_{n-1}: T_{j+1} = 2 y T_j - T_{j-1}
    double T[n][n] = {};
    T[0][0] = 1.0;
    T[1][1] = 1.0;
    for (int j = 1; j + 1 < n; ++j)
        for (int m = 0; m < n; ++m) T[j + 1][m] = (m > 0 ? 2.0 * T[j][m - 1] : 0.0) - T[j - 1][m];
    for (int k = 0; k < K; ++k) {
        const double c = (k + 0.5) * kEwaldH;
        double fa[n], fg[n], y[n];
        for (int i = 0; i < n; ++i) {
            y[i] = std::cos(kPi * (i + 0.5) / n);
            kb_weights_series(S, (c + h * y[i]) / s, &fa[i], &fg[i]);
        }
        for (int w = 0; w < 2; ++w) {
            const double* fv = w == 0 ? fa : fg;
            double b[n];  // Chebyshev coefficients of the interpolant in y = (x - c) / h
            for (int j = 0; j < n; ++j) {
                double acc = 0.0;
                for (int i = 0; i < n; ++i) acc += fv[i] * std::cos(kPi * j * (i + 0.5) / n);
                b[j] = (j == 0 ? 1.0 : 2.0) * acc / n;
            }
            double hm = 1.0;
            for (int m = 0; m < n; ++m) {
                double acc = 0.0;
                for (int j = m; j < n; ++j) acc += b[j] * T[j][m];
                tab[((size_t)w * K + k) * n + m] = acc / hm;
                hm *= h;
            }
        }
    }
}

}  // namespace vpbs

using namespace vpbs;

extern "C" int vpbs_kb_weights(double beta, double rcut, double rtol, const double* r, int64_t n, double* a_table,
                               double* g_table, double* a_series, double* g_series) {
    if (!r || n < 0 || !(beta > 0) || !(rcut > 0) || !(rtol > 0))
        return set_error(nullptr, VPBS_ERR_ARG, "bad arguments");
    const KBSeries S = kb_series(beta, rcut, rtol);
    if (S.f.empty()) return set_error(nullptr, VPBS_ERR_PARAMS, "Kaiser-Bessel series did not converge");
    int K = 0;
    kb_table_host(S, &K, nullptr);
    std::vector<double> tab((size_t)2 * K * kEwaldNC);
    kb_table_host(S, &K, tab.data());
    const double s = kb_table_xmax(beta) / rcut;
    for (int64_t i = 0; i < n; ++i) {
        if (!(r[i] >= 0.0 && r[i] <= rcut)) return set_error(nullptr, VPBS_ERR_ARG, "r outside [0, rcut]");
        double a, g;
        kb_weights_series(S, r[i], &a, &g);
        if (a_series) a_series[i] = a;
        if (g_series) g_series[i] = g;
        const double x = s * r[i];
        int k = (int)(x * kEwaldInvH);
        k = k < K ? k : K - 1;
        const double t = x - (k + 0.5) * kEwaldH;
        const double* ce = tab.data() + (size_t)k * kEwaldNC;
        const double* cg = tab.data() + (size_t)(K + k) * kEwaldNC;
        double ta = ce[kEwaldNC - 1], tg = cg[kEwaldNC - 1];
        for (int m = kEwaldNC - 2; m >= 0; --m) {
            ta = std::fma(ta, t, ce[m]);
            tg = std::fma(tg, t, cg[m]);
        }
        if (a_table) a_table[i] = ta;
        if (g_table) g_table[i] = tg;
    }
    return 0;
}
