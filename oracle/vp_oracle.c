/*
 * vp_oracle.c -- CPU FP64 restatement of VortexPasta's Ewald-split Biot-Savart
 * evaluation on filament nodes.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA library is checked
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.  It is not part of the product library.
 *
 * Parity status: "pinned to the reference's known-answer tests".  The reference is
 * Julia and cannot run here, so there are no reference outputs to compare with;
 * the oracle is instead checked against the analytic ring answers of
 * test/ring.jl, the exact Fourier sums of ExactSumBackend (test/trefoil.jl), exact
 * pair counts (test/cell_lists.jl) and independence from the Ewald parameter
 * alpha and, for the Kaiser-Bessel kernel, from r_cut (test/trefoil.jl:299-329, 422-429).
 *
 * Each function names the reference file:line it restates (paths relative to the
 * VortexPasta.jl tree).  The NUFFT (spreading kernel, oversampled grid size) lives
 * in the external NonuniformFFTs.jl package, which is not part of the reference
 * tree; the oracle uses the published exponential-of-semicircle kernel of Barnett,
 * Magland & af Klinteberg, SIAM J. Sci. Comput. 41 (2019), with its shape
 * parameter beta = 0.97 * pi * (1 - 1/(2 sigma)) * (2m).
 */
#include "vp_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VPO_PI 3.14159265358979323846

typedef double complex cplx;

/* ------------------------------------------------------------------------- */
/* Small vector helpers                                                      */
/* ------------------------------------------------------------------------- */

static inline void cross3(const double* u, const double* v, double* w) {
    /* reference: src/BiotSavart/shortrange/integrands.jl:57-63 */
    w[0] = u[1] * v[2] - u[2] * v[1];
    w[1] = u[2] * v[0] - u[0] * v[2];
    w[2] = u[0] * v[1] - u[1] * v[0];
}

static inline int is_open(const vpo_params* p) { return !(p->L[0] > 0 && p->L[1] > 0 && p->L[2] > 0); }
static inline int ewald_on(const vpo_params* p) { return p->splitting == 1 || p->alpha > 0; }

/* Fold into [0, L).  reference: src/Filaments/min_distance.jl:5-20 (subtraction loops within
 * four periods; one exact fmod beyond, so a huge or non-finite coordinate cannot loop) */
static inline double fold1(double x, double L) {
    if (!(L > 0)) return x;
    if (!(fabs(x) <= 4.0 * L)) {
        x = fmod(x, L);
        if (x < 0) x += L;
        if (x >= L) x = 0.0;
        return x;
    }
    while (x < 0) x += L;
    while (x >= L) x -= L;
    return x;
}

/* Minimum-image separation of two folded coordinates.  reference: min_distance.jl:61-67 */
static inline double deper1(double r, double L) {
    if (!(L > 0)) return r;
    double Lh = 0.5 * L;
    r = (r >= Lh) ? r - L : r;
    r = (r < -Lh) ? r + L : r;
    return r;
}

/* ------------------------------------------------------------------------- */
/* Gauss-Legendre rule on [0,1]  (reference: src/Quadratures/Quadratures.jl)  */
/* ------------------------------------------------------------------------- */

void vpo_gl_rule(int n, double* zeta, double* w) {
    /* Newton iteration on the Legendre polynomial P_n; nodes ascending in [-1,1],
     * then mapped to [0,1] with halved weights (Quadratures.jl:52-56). */
    for (int i = 0; i < n; ++i) {
        double x = cos(VPO_PI * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            double pn = (n == 0) ? 1.0 : (n == 1 ? x : p1);
            double pnm1 = (n == 1) ? 1.0 : p0;
            dp = n * (x * pn - pnm1) / (x * x - 1.0);
            double dx = pn / dp;
            x -= dx;
            if (fabs(dx) < 1e-16) break;
        }
        {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            double pn = (n == 1) ? x : p1;
            double pnm1 = (n == 1) ? 1.0 : p0;
            dp = n * (x * pn - pnm1) / (x * x - 1.0);
        }
        double wi = 2.0 / ((1.0 - x * x) * dp * dp);
        /* i-th root counted from +1 downwards: store ascending */
        zeta[n - 1 - i] = 0.5 * (x + 1.0);
        w[n - 1 - i] = 0.5 * wi;
    }
}

/* ------------------------------------------------------------------------- */
/* Periodic quintic splines with chordal knots                              */
/* reference: src/Filaments/spline/spline.jl:116-139, 264-319,              */
/*            spline/quintic.jl:9-100, parametrisations.jl:43-44,            */
/*            Filaments.jl:695-707                                            */
/* ------------------------------------------------------------------------- */

typedef struct {
    int n;
    double T;          /* knot period */
    double* t;         /* knots t_0..t_{n-1} (t_0 = 0) */
    double* c;         /* [n][3] B-spline coefficients, order 6 */
    double* d1;        /* [n][3] coefficients of s', order 5 */
    double* d2;        /* [n][3] coefficients of s'', order 4 */
    double off[3];     /* end-to-end offset: the curve is y(t) + (t / T) off with y periodic */
} spline_t;

static inline double knot(const spline_t* S, long j) {
    long n = S->n;
    long q = (j >= 0) ? j / n : -((-j + n - 1) / n);
    long r = j - q * n;
    return S->t[r] + (double)q * S->T;
}

static inline long pmod(long j, long n) {
    long r = j % n;
    return r < 0 ? r + n : r;
}

/* de Boor's BSPLVB: values of the k B-splines of order k that are non-zero on
 * [t_i, t_{i+1}), evaluated at x; N[s] = B_{i-k+1+s, k}(x). */
static void bsplvb(const spline_t* S, long i, double x, int k, double* N) {
    double left[8], right[8];
    N[0] = 1.0;
    for (int r = 1; r < k; ++r) {
        left[r] = x - knot(S, i + 1 - r);
        right[r] = knot(S, i + r) - x;
        double saved = 0.0;
        for (int s = 0; s < r; ++s) {
            double tmp = N[s] / (right[s + 1] + left[r - s]);
            N[s] = saved + right[s + 1] * tmp;
            saved = left[r - s] * tmp;
        }
        N[r] = saved;
    }
}

/* Evaluate derivative `der` (0,1,2) of the spline at parameter x within interval i.  With an
 * end-to-end offset the periodic spline y is deperiodised: s = y + (x / T) off, s' = y' + off / T,
 * s'' = y'' (spline.jl:185-194). */
static void spline_eval(const spline_t* S, long i, double x, int der, double* out) {
    int k = 6 - der;
    const double* cs = der == 0 ? S->c : (der == 1 ? S->d1 : S->d2);
    double N[8];
    bsplvb(S, i, x, k, N);
    out[0] = out[1] = out[2] = 0.0;
    for (int s = 0; s < k; ++s) {
        long j = pmod(i - k + 1 + s, S->n);
        for (int d = 0; d < 3; ++d) out[d] += cs[3 * j + d] * N[s];
    }
    if (der == 0)
        for (int d = 0; d < 3; ++d) out[d] += (x / S->T) * S->off[d];
    else if (der == 1)
        for (int d = 0; d < 3; ++d) out[d] += S->off[d] / S->T;
}

/* Evaluate at local coordinate zeta in [0,1] on segment i (spline.jl:116-124). */
static void spline_eval_seg(const spline_t* S, long i, double zeta, int der, double* out) {
    double ti = knot(S, i), ti1 = knot(S, i + 1);
    double x = (1.0 - zeta) * ti + zeta * ti1;
    spline_eval(S, i, x, der, out);
}

/* Solve a 4x4 system H s = r (3 right-hand sides) with partial pivoting. */
static int solve4(double H[4][4], double r[4][3]) {
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int i = c + 1; i < 4; ++i)
            if (fabs(H[i][c]) > fabs(H[piv][c])) piv = i;
        if (H[piv][c] == 0.0) return -1;
        if (piv != c) {
            for (int j = 0; j < 4; ++j) { double t = H[c][j]; H[c][j] = H[piv][j]; H[piv][j] = t; }
            for (int j = 0; j < 3; ++j) { double t = r[c][j]; r[c][j] = r[piv][j]; r[piv][j] = t; }
        }
        for (int i = c + 1; i < 4; ++i) {
            double f = H[i][c] / H[c][c];
            for (int j = c; j < 4; ++j) H[i][j] -= f * H[c][j];
            for (int j = 0; j < 3; ++j) r[i][j] -= f * r[c][j];
        }
    }
    for (int c = 3; c >= 0; --c) {
        for (int j = 0; j < 3; ++j) {
            double s = r[c][j];
            for (int k = c + 1; k < 4; ++k) s -= H[c][k] * r[k][j];
            r[c][j] = s / H[c][c];
        }
    }
    return 0;
}

/* Build the periodic quintic interpolating spline through X_0..X_{n-1} (closed curve; with an
 * end-to-end offset `off` (NULL: zero) the node after X_{n-1} is X_0 + off, the chordal knots
 * include that closing segment and the periodic spline interpolates y_i = X_i - (t_i / T) off,
 * closed_filament.jl:196-207, spline.jl:163-182, quintic.jl:9-17).
 * The cyclic pentadiagonal collocation system is split as A = B + U W with B the
 * (non-cyclic) pentadiagonal part and U W the four wrap-around corner rows; B is
 * factorised by banded elimination without pivoting (B-spline collocation matrices
 * are totally positive) and the corners are handled with the Woodbury identity. */
static int spline_build(spline_t* S, int n, const double* X, const double* off) {
    if (n < 5) return -1;
    S->n = n;
    for (int d = 0; d < 3; ++d) S->off[d] = off ? off[d] : 0.0;
    S->t = (double*)malloc(sizeof(double) * n);
    S->c = (double*)malloc(sizeof(double) * 3 * n);
    S->d1 = (double*)malloc(sizeof(double) * 3 * n);
    S->d2 = (double*)malloc(sizeof(double) * 3 * n);
    /* chordal knots */
    double t = 0.0;
    for (int i = 0; i < n; ++i) {
        S->t[i] = t;
        int j = (i + 1) % n;
        double e[3];
        for (int d = 0; d < 3; ++d) e[d] = X[3 * j + d] + (j == 0 ? S->off[d] : 0.0) - X[3 * i + d];
        t += sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    }
    S->T = t;

    /* collocation rows: row i has B_{i-5..i-1,6}(t_i) on unknowns u_{i-2..i+2} */
    double* band = (double*)calloc((size_t)5 * n, sizeof(double)); /* band[i*5 + (o+2)] */
    double W[4][8];   /* corner values */
    int Wc[4][2];     /* corner columns */
    int nW[4] = {0, 0, 0, 0};
    const int Urow[4] = {0, 1, n - 2, n - 1};
    for (int i = 0; i < n; ++i) {
        double N[8];
        bsplvb(S, i, knot(S, i), 6, N);
        for (int s = 0; s < 5; ++s) {
            int o = s - 2;
            int col = i + o;
            if (col >= 0 && col < n) {
                band[i * 5 + (o + 2)] += N[s];
            } else {
                int cw = (int)pmod(col, n);
                int r = (i == 0) ? 0 : (i == 1) ? 1 : (i == n - 2) ? 2 : 3;
                W[r][nW[r]] = N[s];
                Wc[r][nW[r]] = cw;
                nW[r]++;
            }
        }
    }
    /* banded LU (no pivoting): multipliers stored in the sub-diagonal slots */
    for (int i = 0; i < n; ++i) {
        double piv = band[i * 5 + 2];
        for (int r = i + 1; r <= i + 2 && r < n; ++r) {
            double f = band[r * 5 + (i - r + 2)] / piv;
            band[r * 5 + (i - r + 2)] = f;
            for (int c = i + 1; c <= i + 2 && c < n; ++c) band[r * 5 + (c - r + 2)] -= f * band[i * 5 + (c - i + 2)];
        }
    }
    /* right-hand sides: 3 coordinates + 4 columns of U */
    double* Y = (double*)malloc(sizeof(double) * 7 * n);
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) Y[7 * i + d] = X[3 * i + d] - (S->t[i] / S->T) * S->off[d];
        for (int q = 0; q < 4; ++q) Y[7 * i + 3 + q] = (i == Urow[q]) ? 1.0 : 0.0;
    }
    for (int i = 0; i < n; ++i)          /* forward (unit lower) */
        for (int r = i + 1; r <= i + 2 && r < n; ++r) {
            double f = band[r * 5 + (i - r + 2)];
            for (int q = 0; q < 7; ++q) Y[7 * r + q] -= f * Y[7 * i + q];
        }
    for (int i = n - 1; i >= 0; --i) {   /* backward (upper) */
        for (int c = i + 1; c <= i + 2 && c < n; ++c) {
            double u = band[i * 5 + (c - i + 2)];
            for (int q = 0; q < 7; ++q) Y[7 * i + q] -= u * Y[7 * c + q];
        }
        for (int q = 0; q < 7; ++q) Y[7 * i + q] /= band[i * 5 + 2];
    }
    /* Woodbury: H = I + W Z, rhs = W y; x = y - Z H^{-1} W y */
    double H[4][4], rh[4][3];
    for (int r = 0; r < 4; ++r) {
        for (int q = 0; q < 4; ++q) H[r][q] = (r == q) ? 1.0 : 0.0;
        for (int d = 0; d < 3; ++d) rh[r][d] = 0.0;
        for (int e = 0; e < nW[r]; ++e) {
            int col = Wc[r][e];
            for (int q = 0; q < 4; ++q) H[r][q] += W[r][e] * Y[7 * col + 3 + q];
            for (int d = 0; d < 3; ++d) rh[r][d] += W[r][e] * Y[7 * col + d];
        }
    }
    int err = solve4(H, rh);
    double* u = (double*)malloc(sizeof(double) * 3 * n);
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            double s = Y[7 * i + d];
            for (int q = 0; q < 4; ++q) s -= Y[7 * i + 3 + q] * rh[q][d];
            u[3 * i + d] = s;
        }
    /* c_j = u_{j+3} */
    for (int j = 0; j < n; ++j)
        for (int d = 0; d < 3; ++d) S->c[3 * j + d] = u[3 * pmod(j + 3, n) + d];
    /* derivative coefficients (spline.jl:301-319 for the recurrence) */
    for (int j = 0; j < n; ++j) {
        long jm = pmod(j - 1, n);
        double den = knot(S, j + 5) - knot(S, j);
        for (int d = 0; d < 3; ++d) S->d1[3 * j + d] = 5.0 * (S->c[3 * j + d] - S->c[3 * jm + d]) / den;
    }
    for (int j = 0; j < n; ++j) {
        long jm = pmod(j - 1, n);
        double den = knot(S, j + 4) - knot(S, j);
        for (int d = 0; d < 3; ++d) S->d2[3 * j + d] = 4.0 * (S->d1[3 * j + d] - S->d1[3 * jm + d]) / den;
    }
    free(u);
    free(Y);
    free(band);
    return err;
}

static void spline_free(spline_t* S) {
    free(S->t); free(S->c); free(S->d1); free(S->d2);
}

/* ------------------------------------------------------------------------- */
/* Point data  (reference: src/BiotSavart/pointdata_impl.jl:41-108)          */
/* ------------------------------------------------------------------------- */

static double seg_length(const spline_t* S, long i, int nq, const double* zq, const double* wq, double a, double b) {
    double dt = knot(S, i + 1) - knot(S, i);
    double acc = 0.0;
    for (int q = 0; q < nq; ++q) {
        double d[3];
        spline_eval_seg(S, i, a + (b - a) * zq[q], 1, d);
        acc += wq[q] * sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
    return dt * (b - a) * acc;
}

static void filament_point_data(const vpo_params* p, const spline_t* S, const double* X, int64_t off,
                                const double* zq, const double* wq,
                                double* nodes_f, int32_t* idx_prev, double* d1, double* d2,
                                double* dm, double* dp, double* points, double* charges) {
    int n = S->n, nq = p->nquad;
    double g = p->lia_segment_fraction;
    int has_g = g > 0;
    for (int i = 0; i < n; ++i) {
        int64_t k = off + i;
        for (int d = 0; d < 3; ++d) nodes_f[3 * k + d] = fold1(X[3 * i + d], p->L[d]);
        idx_prev[k] = (int32_t)(i == 0 ? off + n - 1 : k - 1);
        spline_eval_seg(S, i, 0.0, 1, d1 + 3 * k);
        spline_eval_seg(S, i, 0.0, 2, d2 + 3 * k);
        /* lia_integration_limits: ((1-g, 1), (0, g))  (local_integrals.jl:100-101) */
        dm[k] = seg_length(S, i - 1, nq, zq, wq, has_g ? 1.0 - g : 0.0, 1.0);
        dp[k] = seg_length(S, i, nq, zq, wq, 0.0, has_g ? g : 1.0);
        double dt = knot(S, i + 1) - knot(S, i);
        for (int q = 0; q < nq; ++q) {
            int64_t mq = k * nq + q;
            double s[3], sp[3];
            spline_eval_seg(S, i, zq[q], 0, s);
            spline_eval_seg(S, i, zq[q], 1, sp);
            for (int d = 0; d < 3; ++d) {
                points[3 * mq + d] = fold1(s[d], p->L[d]);
                charges[3 * mq + d] = wq[q] * dt * sp[d];
            }
        }
    }
}

int vpo_point_data(const vpo_params* p, int nfil, const int64_t* offsets, const double* nodes_xyz,
                   double* nodes_f, int32_t* idx_prev, double* d1, double* d2,
                   double* dm, double* dp, double* points, double* charges) {
    double zq[32], wq[32];
    if (p->nquad < 1 || p->nquad > 32) return -1;
    vpo_gl_rule(p->nquad, zq, wq);
    int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
    for (int f = 0; f < nfil; ++f) {
        int64_t off = offsets[f];
        int n = (int)(offsets[f + 1] - off);
        spline_t S;
        if (spline_build(&S, n, nodes_xyz + 3 * off, p->fil_offsets ? p->fil_offsets + 3 * f : NULL) != 0) {
            err |= 1;
            continue;
        }
        filament_point_data(p, &S, nodes_xyz + 3 * off, off, zq, wq, nodes_f, idx_prev, d1, d2, dm, dp, points, charges);
        spline_free(&S);
    }
    return err ? -2 : 0;
}

/* ------------------------------------------------------------------------- */
/* Local term and self-interaction removal                                   */
/* reference: src/BiotSavart/shortrange/local_integrals.jl:4-165             */
/* ------------------------------------------------------------------------- */

static void local_term(const vpo_params* p, int64_t Np, const double* d1, const double* d2,
                       const double* dm, const double* dp, double* vel, double* psi) {
    double pref = p->Gamma / (4.0 * VPO_PI);
    double rpsi = exp(p->Delta - 1.0) * p->a / 2.0;
    double rv = rpsi * exp(1.0);
#pragma omp parallel for
    for (int64_t i = 0; i < Np; ++i) {
        double delta = sqrt(dm[i] * dp[i]);
        const double* s1 = d1 + 3 * i;
        const double* s2 = d2 + 3 * i;
        double mu2 = s1[0] * s1[0] + s1[1] * s1[1] + s1[2] * s1[2];
        double mu_inv = 1.0 / sqrt(mu2);
        if (vel) {
            double b[3];
            cross3(s1, s2, b);
            double f = log(delta / rv) * mu_inv * mu_inv * mu_inv;
            for (int d = 0; d < 3; ++d) vel[3 * i + d] = pref * (f * b[d]);
        }
        if (psi) {
            double f = 2.0 * log(delta / rpsi) * mu_inv;
            for (int d = 0; d < 3; ++d) psi[3 * i + d] = pref * (f * s1[d]);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Kaiser-Bessel splitting: src/BiotSavart/splitting/kaiser_bessel.jl,       */
/*                          src/BiotSavart/splitting/chebyshev.jl            */
/* ------------------------------------------------------------------------- */

/* Modified Bessel function I0 by its power series sum_k (z^2/4)^k / (k!)^2 (all terms positive,
 * so summing until the term no longer changes the sum is accurate to rounding). */
static double bessel_i0(double z) {
    double q = 0.25 * z * z, term = 1.0, sum = 1.0;
    for (int k = 1; k < 500; ++k) {
        term *= q / ((double)k * k);
        double s2 = sum + term;
        if (s2 == sum) break;
        sum = s2;
    }
    return sum;
}

typedef struct {
    double rcut;
    int ne;          /* even coefficients of f: T_0, T_2, ..., T_{2(ne-1)} */
    double* fe;
    double* Fo;      /* odd coefficients of F: T_1, T_3, ..., T_{2 ne - 1} */
} kb_series;

/* chebyshev.jl:130-172 (approximate, symmetry = :even): values of
 * f(r) = beta / (rcut sinh beta) I0(beta sqrt(1 - r^2/rcut^2)) on r_n = rcut cos(pi n/(N-1)),
 * FFTW's REDFT00 (type-I DCT) written out, ends halved, / (N - 1); truncation before the first
 * pair of consecutive coefficients below rtol * sum|c| (N doubles from 64 otherwise); the
 * even-index coefficients before it are kept.  Then chebyshev.jl:99-122 (integrate even -> odd,
 * times rcut). */
static int kb_build(double beta, double rcut, double rtol, kb_series* S) {
    S->rcut = rcut;
    S->ne = 0;
    S->fe = S->Fo = NULL;
    double C = beta / (rcut * sinh(beta));
    for (int N = 64; N <= 4096; N *= 2) {
        double* u = (double*)malloc(sizeof(double) * N);
        double* c = (double*)malloc(sizeof(double) * N);
        for (int n = 0; n < N; ++n) {
            double x = rcut * cos(VPO_PI * n / (N - 1));
            double t = 1.0 - (x / rcut) * (x / rcut);
            u[n] = C * bessel_i0(beta * sqrt(t > 0 ? t : 0.0));
        }
        double total = 0.0;
        for (int k = 0; k < N; ++k) {
            double y = u[0] + ((k & 1) ? -u[N - 1] : u[N - 1]);
            for (int j = 1; j < N - 1; ++j) {
                long ph = ((long)j * k) % (2L * (N - 1));
                y += 2.0 * u[j] * cos(VPO_PI * (double)ph / (N - 1));
            }
            if (k == 0 || k == N - 1) y *= 0.5;
            c[k] = y / (N - 1);
            total += fabs(c[k]);
        }
        double atol = rtol * total;
        int cut = -1;
        for (int j = 0; j + 1 < N; ++j)
            if (fabs(c[j]) < atol && fabs(c[j + 1]) < atol) { cut = j; break; }
        free(u);
        if (cut >= 1) {
            int ne = (cut + 1) / 2;  /* even indices 0, 2, ..., < cut */
            S->ne = ne;
            S->fe = (double*)malloc(sizeof(double) * ne);
            S->Fo = (double*)malloc(sizeof(double) * ne);
            for (int i = 0; i < ne; ++i) S->fe[i] = c[2 * i];
            free(c);
            if (ne == 1) {
                S->Fo[0] = S->fe[0];
            } else {
                S->Fo[0] = (2.0 * S->fe[0] - S->fe[1]) / 2.0;
                for (int i = 1; i < ne - 1; ++i) S->Fo[i] = (S->fe[i] - S->fe[i + 1]) / (2.0 * (2 * i + 1));
                S->Fo[ne - 1] = S->fe[ne - 1] / (2.0 * (2 * ne - 1));
            }
            for (int i = 0; i < ne; ++i) S->Fo[i] *= rcut;
            return 0;
        }
        free(c);
    }
    return -1;
}

static void kb_free(kb_series* S) {
    free(S->fe);
    free(S->Fo);
    S->fe = S->Fo = NULL;
    S->ne = 0;
}

/* chebyshev.jl:50-71: Clenshaw recurrences of the even and odd series (x = r / rcut). */
static double cheb_even(const double* cs, int N, double x) {
    double bpp = 0.0, bp = 0.0, twox = 2.0 * x;
    for (int n = N - 1; n >= 1; --n) {
        double b = twox * bp + cs[n] - bpp;
        bpp = bp; bp = b;
        b = twox * bp - bpp;
        bpp = bp; bp = b;
    }
    return cs[0] + x * bp - bpp;
}

static double cheb_odd(const double* cs, int N, double x) {
    double bpp = 0.0, bp = cs[N - 1], twox = 2.0 * x;
    for (int n = N - 2; n >= 0; --n) {
        double b = twox * bp - bpp;
        bpp = bp; bp = b;
        b = twox * bp + cs[n] - bpp;
        bpp = bp; bp = b;
    }
    return x * bp - bpp;
}

/* weights_shortrange (kaiser_bessel.jl:282-292): a = 1 - F(r), b = r f(r) */
static inline void kb_short_weights(const kb_series* S, double r, double* a, double* b) {
    double x = r / S->rcut;
    *a = 1.0 - cheb_odd(S->Fo, S->ne, x);
    *b = r * cheb_even(S->fe, S->ne, x);
}

/* splitting_kernel_fourier (kaiser_bessel.jl:266-278) */
static inline double kb_fourier(double beta, double rcut, double k2) {
    double s = beta * beta - k2 * rcut * rcut;
    if (!(s > 0)) return 0.0;
    double q = sqrt(s);
    return beta / sinh(beta) * sinh(q) / q;
}

/* The series of the current call (built once per vpo_compute_on_nodes). */
static kb_series g_kb;

int vpo_kb_weights(double beta, double rcut, double rtol, const double* r, long n, double* a, double* g) {
    kb_series S;
    if (kb_build(beta, rcut, rtol, &S)) return -1;
    for (long i = 0; i < n; ++i) {
        double wa, wb;
        kb_short_weights(&S, r[i], &wa, &wb);
        a[i] = wa;
        g[i] = wa + wb;
    }
    int ne = S.ne;
    kb_free(&S);
    return ne;
}

static void remove_self(const vpo_params* p, int64_t Np, const double* nodes_f, const int32_t* idx_prev,
                        const double* points, const double* charges, double* vel, double* psi) {
    double pref = p->Gamma / (4.0 * VPO_PI);
    int nq = p->nquad;
    double alpha = p->alpha;
    int explicit_erf = !p->avoid_explicit_erf && ewald_on(p);
#pragma omp parallel for
    for (int64_t i = 0; i < Np; ++i) {
        const double* x = nodes_f + 3 * i;
        int64_t ip = idx_prev[i];
        for (int side = 0; side < 2; ++side) {
            int64_t base = (side == 0 ? ip : i) * nq;
            for (int q = 0; q < nq; ++q) {
                int64_t j = base + q;
                double r[3];
                for (int d = 0; d < 3; ++d) r[d] = deper1(x[d] - points[3 * j + d], p->L[d]);
                double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                double rr = sqrt(r2);
                double rinv = 1.0 / rr;
                const double* qc = charges + 3 * j;
                double fa = 1.0, fb = 0.0;
                if (explicit_erf && p->splitting == 1) {
                    /* weights_longrange (kaiser_bessel.jl:296-301): (F, r f) inside rcut, (1, 0) beyond */
                    if (rr < p->rcut) {
                        double sa, sb;
                        kb_short_weights(&g_kb, rr, &sa, &sb);
                        fa = 1.0 - sa;
                        fb = sb;
                    }
                } else if (explicit_erf) {
                    double ar = alpha * rr;
                    fa = erf(ar);
                    fb = 2.0 / sqrt(VPO_PI) * ar * exp(-(ar * ar));
                }
                if (vel) {
                    double c[3];
                    cross3(qc, r, c);
                    double f = explicit_erf ? (fa - fb) * rinv * rinv * rinv : rinv * rinv * rinv;
                    for (int d = 0; d < 3; ++d) vel[3 * i + d] -= pref * (f * c[d]);
                }
                if (psi) {
                    double f = explicit_erf ? fa * rinv : rinv;
                    for (int d = 0; d < 3; ++d) psi[3 * i + d] -= pref * (f * qc[d]);
                }
            }
        }
    }
}

/* add_local_integrals! for lia_segment_fraction (local_integrals.jl:209-305) */
static void local_integrals(const vpo_params* p, const spline_t* S, int64_t off, const double* nodes_f,
                            double* vel, double* psi) {
    double g = p->lia_segment_fraction;
    int nq = p->nquad_near > 0 ? p->nquad_near : p->nquad;
    double zq[32], wq[32];
    vpo_gl_rule(nq, zq, wq);
    double pref = p->Gamma / (4.0 * VPO_PI);
    for (int i = 0; i < S->n; ++i) {
        int64_t k = off + i;
        const double* x = nodes_f + 3 * k;
        double dv[3] = {0, 0, 0}, dpsi[3] = {0, 0, 0};
        for (int side = 0; side < 2; ++side) {
            long seg = side == 0 ? i - 1 : i;
            double a = side == 0 ? 0.0 : g, b = side == 0 ? 1.0 - g : 1.0;
            double dt = (knot(S, seg + 1) - knot(S, seg)) * (b - a);
            for (int q = 0; q < nq; ++q) {
                double y = a + (b - a) * zq[q];
                double s[3], sp[3], r[3], qc[3];
                spline_eval_seg(S, seg, y, 0, s);
                spline_eval_seg(S, seg, y, 1, sp);
                for (int d = 0; d < 3; ++d) {
                    qc[d] = wq[q] * dt * sp[d];
                    r[d] = deper1(x[d] - fold1(s[d], p->L[d]), p->L[d]);
                }
                double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                double rinv = 1.0 / rr;
                double c[3];
                cross3(qc, r, c);
                for (int d = 0; d < 3; ++d) {
                    dv[d] += rinv * rinv * rinv * c[d];
                    dpsi[d] += rinv * qc[d];
                }
            }
        }
        for (int d = 0; d < 3; ++d) {
            if (vel) vel[3 * k + d] += pref * dv[d];
            if (psi) psi[3 * k + d] += pref * dpsi[d];
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Short-range pair interactions                                             */
/* reference: src/BiotSavart/shortrange/shortrange.jl:216-273,               */
/*            integrands.jl:2-18, splitting/gaussian.jl:273-279,             */
/*            src/CellLists/CellLists.jl:117-163, 194-204, 384-434           */
/* ------------------------------------------------------------------------- */

typedef struct {
    double v[3], psi[3];
    int64_t inrange, cand;
} pair_acc;

static inline void pair_one(const vpo_params* p, const double* x, const double* s, const double* qc,
                            double rcut2, int want_v, int want_psi, pair_acc* acc) {
    double r[3];
    for (int d = 0; d < 3; ++d) r[d] = deper1(x[d] - s[d], p->L[d]);
    double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    acc->cand++;
    if (!(r2 <= rcut2)) return;
    acc->inrange++;
    double rr = sqrt(r2);
    double rinv = 1.0 / rr;
    double a = 1.0, b = 0.0;
    if (p->splitting == 1) {
        kb_short_weights(&g_kb, rr, &a, &b);
    } else if (p->alpha > 0) {
        double ar = p->alpha * rr;
        a = erfc(ar);
        b = 2.0 / sqrt(VPO_PI) * ar * exp(-(ar * ar));
    }
    if (want_v) {
        double c[3];
        cross3(qc, r, c);
        double f = (a + b) * rinv * rinv * rinv;
        for (int d = 0; d < 3; ++d) acc->v[d] += f * c[d];
    }
    if (want_psi) {
        double f = a * rinv;
        for (int d = 0; d < 3; ++d) acc->psi[d] += f * qc[d];
    }
}

static inline int is_local_pair(int64_t i, int64_t ip, int64_t j, int nq) {
    return (j / nq == i) || (j / nq == ip);
}

static void pairs(const vpo_params* p, int64_t Np, int64_t Nq, const double* nodes_f, const int32_t* idx_prev,
                  const double* points, const double* charges, double* vel, double* psi, vpo_stats* st) {
    double pref = p->Gamma / (4.0 * VPO_PI);
    double rcut2 = ewald_on(p) ? p->rcut * p->rcut : INFINITY;
    int want_v = vel != NULL, want_psi = psi != NULL;
    int skip_local = !p->avoid_explicit_erf && ewald_on(p);
    int nq = p->nquad;
    int64_t tot_in = 0, tot_cand = 0;
    int M = p->nsubdiv;
    if (M <= 0 || is_open(p) || !ewald_on(p)) {
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tot_in, tot_cand)
        for (int64_t i = 0; i < Np; ++i) {
            pair_acc acc;
            memset(&acc, 0, sizeof acc);
            for (int64_t j = 0; j < Nq; ++j) {
                if (skip_local && is_local_pair(i, idx_prev[i], j, nq)) continue;
                pair_one(p, nodes_f + 3 * i, points + 3 * j, charges + 3 * j, rcut2, want_v, want_psi, &acc);
            }
            for (int d = 0; d < 3; ++d) {
                if (want_v) vel[3 * i + d] += pref * acc.v[d];
                if (want_psi) psi[3 * i + d] += pref * acc.psi[d];
            }
            tot_in += acc.inrange;
            tot_cand += acc.cand;
        }
    } else {
        /* cell lists: nc = floor(L*M/rcut) cells per direction (CellLists.jl:140-145),
         * counting sort of the sources by cell, (2M+1)^3 neighbour cells per node. */
        int nc[3];
        for (int d = 0; d < 3; ++d) nc[d] = (int)floor(p->L[d] * M / p->rcut);
        int64_t ncell = (int64_t)nc[0] * nc[1] * nc[2];
        int64_t* start = (int64_t*)calloc((size_t)ncell + 1, sizeof(int64_t));
        int64_t* cellof = (int64_t*)malloc(sizeof(int64_t) * (Nq > 0 ? Nq : 1));
        int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (Nq > 0 ? Nq : 1));
        for (int64_t j = 0; j < Nq; ++j) {
            int ci[3];
            for (int d = 0; d < 3; ++d) {
                ci[d] = (int)(points[3 * j + d] / p->L[d] * nc[d]);
                if (ci[d] >= nc[d]) ci[d] = nc[d] - 1;
                if (ci[d] < 0) ci[d] = 0;
            }
            cellof[j] = ((int64_t)ci[2] * nc[1] + ci[1]) * nc[0] + ci[0];
            start[cellof[j] + 1]++;
        }
        for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
        {
            int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncell);
            memcpy(fill, start, sizeof(int64_t) * (size_t)ncell);
            for (int64_t j = 0; j < Nq; ++j) order[fill[cellof[j]]++] = j;
            free(fill);
        }
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tot_in, tot_cand)
        for (int64_t i = 0; i < Np; ++i) {
            const double* x = nodes_f + 3 * i;
            int ci[3];
            for (int d = 0; d < 3; ++d) {
                ci[d] = (int)(x[d] / p->L[d] * nc[d]);
                if (ci[d] >= nc[d]) ci[d] = nc[d] - 1;
                if (ci[d] < 0) ci[d] = 0;
            }
            pair_acc acc;
            memset(&acc, 0, sizeof acc);
            for (int dz = -M; dz <= M; ++dz)
                for (int dy = -M; dy <= M; ++dy)
                    for (int dx = -M; dx <= M; ++dx) {
                        int64_t cz = pmod(ci[2] + dz, nc[2]), cy = pmod(ci[1] + dy, nc[1]), cx = pmod(ci[0] + dx, nc[0]);
                        int64_t c = (cz * nc[1] + cy) * nc[0] + cx;
                        for (int64_t t = start[c]; t < start[c + 1]; ++t) {
                            int64_t j = order[t];
                            if (skip_local && is_local_pair(i, idx_prev[i], j, nq)) continue;
                            pair_one(p, x, points + 3 * j, charges + 3 * j, rcut2, want_v, want_psi, &acc);
                        }
                    }
            for (int d = 0; d < 3; ++d) {
                if (want_v) vel[3 * i + d] += pref * acc.v[d];
                if (want_psi) psi[3 * i + d] += pref * acc.psi[d];
            }
            tot_in += acc.inrange;
            tot_cand += acc.cand;
        }
        free(start); free(cellof); free(order);
    }
    if (st) {
        st->pairs_in_range = tot_in;
        st->pairs_candidates = tot_cand;
    }
}

/* ------------------------------------------------------------------------- */
/* FFT (mixed radix 2/3/5, complex, unnormalised)                            */
/* ------------------------------------------------------------------------- */

int vpo_fft_size(int Ns, double sigma) {
    int n = (int)ceil(sigma * Ns - 1e-9);
    if (n < 2) n = 2;
    for (;; ++n) {
        if (n % 2) continue;
        int r = n;
        while (r % 2 == 0) r /= 2;
        while (r % 3 == 0) r /= 3;
        while (r % 5 == 0) r /= 5;
        if (r == 1) return n;
    }
}

typedef struct {
    int n;
    int nf;
    int fac[32];
    cplx* tw; /* e^{sign 2 pi i j/n} */
} fftplan;

static void fft_plan_init(fftplan* P, int n, int sign) {
    P->n = n;
    P->nf = 0;
    int r = n;
    const int rad[3] = {2, 3, 5};
    for (int k = 0; k < 3; ++k)
        while (r % rad[k] == 0) { P->fac[P->nf++] = rad[k]; r /= rad[k]; }
    P->tw = (cplx*)malloc(sizeof(cplx) * n);
    for (int j = 0; j < n; ++j) P->tw[j] = cexp(sign * 2.0 * VPO_PI * I * j / n);
}

/* out[0..n) = DFT of in[0, is, 2is, ...] (decimation in time, recursive). */
static void fft_rec(const fftplan* P, int n, int depth, const cplx* in, long is, cplx* out, int twstride) {
    if (n == 1) { out[0] = in[0]; return; }
    int p = P->fac[depth];
    int m = n / p;
    for (int q = 0; q < p; ++q) fft_rec(P, m, depth + 1, in + q * is, is * p, out + q * m, twstride * p);
    cplx tmp[5];
    for (int k = 0; k < m; ++k) {
        for (int q = 0; q < p; ++q) tmp[q] = out[q * m + k] * P->tw[((long)q * k * twstride) % P->n];
        for (int q2 = 0; q2 < p; ++q2) {
            cplx s = 0;
            for (int q = 0; q < p; ++q) s += tmp[q] * P->tw[((long)q * q2 * m * twstride) % P->n];
            out[q2 * m + k] = s;
        }
    }
}

/* In-place 3-D complex FFT of a [n2][n1][n0] array (x fastest). */
static void fft3(cplx* a, const int n[3], int sign) {
    fftplan P[3];
    for (int d = 0; d < 3; ++d) fft_plan_init(&P[d], n[d], sign);
    long n0 = n[0], n1 = n[1], n2 = n[2];
    /* x lines */
#pragma omp parallel
    {
        int nmax = n0 > n1 ? (n0 > n2 ? n0 : n2) : (n1 > n2 ? n1 : n2);
        cplx* bin = (cplx*)malloc(sizeof(cplx) * nmax);
        cplx* bout = (cplx*)malloc(sizeof(cplx) * nmax);
#pragma omp for
        for (long l = 0; l < n1 * n2; ++l) {
            cplx* line = a + l * n0;
            memcpy(bin, line, sizeof(cplx) * n0);
            fft_rec(&P[0], (int)n0, 0, bin, 1, bout, 1);
            memcpy(line, bout, sizeof(cplx) * n0);
        }
#pragma omp for
        for (long l = 0; l < n0 * n2; ++l) {
            long ix = l % n0, iz = l / n0;
            for (long iy = 0; iy < n1; ++iy) bin[iy] = a[(iz * n1 + iy) * n0 + ix];
            fft_rec(&P[1], (int)n1, 0, bin, 1, bout, 1);
            for (long iy = 0; iy < n1; ++iy) a[(iz * n1 + iy) * n0 + ix] = bout[iy];
        }
#pragma omp for
        for (long l = 0; l < n0 * n1; ++l) {
            for (long iz = 0; iz < n2; ++iz) bin[iz] = a[iz * n0 * n1 + l];
            fft_rec(&P[2], (int)n2, 0, bin, 1, bout, 1);
            for (long iz = 0; iz < n2; ++iz) a[iz * n0 * n1 + l] = bout[iz];
        }
        free(bin);
        free(bout);
    }
    for (int d = 0; d < 3; ++d) free(P[d].tw);
}

/* ------------------------------------------------------------------------- */
/* Long range  (reference: src/BiotSavart/longrange/longrange.jl:102-156,     */
/*   380-471, 488-583; backends/nonuniformffts.jl:153-212;                  */
/*   backends/exact_sum.jl:72-121; cache_common.jl:64-108)                  */
/* ------------------------------------------------------------------------- */

/* Spreading kernels: ES (exponential of semicircle, Barnett, Magland & af Klinteberg 2019) with
 * beta = 0.97 pi m (2 - 1/sigma), or the backward Kaiser-Bessel kernel of the NFFT literature
 * (Potts & Steidl 2003) with beta = 0.995 pi m (2 - 1/sigma); p->nufft_kernel selects (0 / 1). */
static double es_beta(const vpo_params* p) {
    if (p->nufft_kernel == 1) return 0.995 * VPO_PI * p->m * (2.0 - 1.0 / p->sigma);
    return 0.97 * VPO_PI * (1.0 - 1.0 / (2.0 * p->sigma)) * (2.0 * p->m);
}
static int g_kernel_kind = 0; /* kernel of the current evaluation (set with the parameters) */

/* Kernels shifted down by their edge value, so that they vanish continuously at |u| = m: the
 * 2m-point window of a point lying on a grid node then does not depend on the last bit of its
 * coordinate.  With r = sqrt(1 - (u/m)^2): ES exp(beta (r - 1)) - e^{-beta}; backward
 * Kaiser-Bessel sinh(beta r) / (r sinh beta) - beta / sinh beta. */
static inline double es_kernel(double u, int m, double beta) {
    double z = u / m;
    double s = 1.0 - z * z;
    if (!(s > 0)) return 0.0;
    if (g_kernel_kind == 1) {
        double r = sqrt(s);
        return (r > 1e-12 ? sinh(beta * r) / (r * sinh(beta)) : beta / sinh(beta)) - beta / sinh(beta);
    }
    return exp(beta * (sqrt(s) - 1.0)) - exp(-beta);
}

/* Fourier transform of the (shifted) ES kernel in grid units: int_{-m}^{m} psi(u) cos(xi u) du,
 * via u = m sin(theta) and a 128-point Gauss-Legendre rule on [-pi/2, pi/2]. */
static double es_hat(double xi, int m, double beta) {
    static __thread double gz[128], gw[128];
    static __thread int init = 0;
    if (!init) {
        double z01[128], w01[128];
        vpo_gl_rule(128, z01, w01);
        for (int i = 0; i < 128; ++i) { gz[i] = VPO_PI * (z01[i] - 0.5); gw[i] = VPO_PI * w01[i]; }
        init = 1;
    }
    double s = 0.0;
    for (int i = 0; i < 128; ++i) {
        double th = gz[i];
        double c = cos(th);
        double pc = g_kernel_kind == 1 ? sinh(beta * c) / sinh(beta) - (beta / sinh(beta)) * c
                                       : (exp(beta * (c - 1.0)) - exp(-beta)) * c;
        s += gw[i] * pc * cos(xi * m * sin(th));
    }
    return m * s;
}

static inline int mode_of(int i, int N) { return i < (N + 1) / 2 ? i : i - N; }

typedef struct {
    int Ns[3];
    int nkx;             /* Ns0/2 + 1 */
    double* uhat;        /* [3][Ns2][Ns1][nkx] complex interleaved */
    double k0[3];        /* 2 pi / L */
} lr_field;

static inline size_t uidx(const lr_field* F, int c, int ix, int iy, int iz) {
    return (((size_t)c * F->Ns[2] + iz) * F->Ns[1] + iy) * F->nkx + ix;
}

/* Hermitian-symmetry zeroing (longrange.jl:556-583). */
static void ensure_hermitian(lr_field* F) {
    for (int c = 0; c < 3; ++c)
        for (int iz = 0; iz < F->Ns[2]; ++iz)
            for (int iy = 0; iy < F->Ns[1]; ++iy)
                for (int ix = 0; ix < F->nkx; ++ix) {
                    int zero = (ix == F->nkx - 1);
                    if (F->Ns[1] % 2 == 0 && iy == F->Ns[1] / 2) zero = 1;
                    if (F->Ns[2] % 2 == 0 && iz == F->Ns[2] / 2) zero = 1;
                    if (zero) {
                        size_t u = uidx(F, c, ix, iy, iz);
                        F->uhat[2 * u] = F->uhat[2 * u + 1] = 0.0;
                    }
                }
}

static void truncate_spherical(const vpo_params* p, lr_field* F) {
    double kmax = INFINITY;
    for (int d = 0; d < 3; ++d) {
        double km = 2.0 * VPO_PI * ((F->Ns[d] - 1) / 2) / p->L[d];
        if (km < kmax) kmax = km;
    }
    double kmax2 = kmax * kmax;
    for (int iz = 0; iz < F->Ns[2]; ++iz)
        for (int iy = 0; iy < F->Ns[1]; ++iy)
            for (int ix = 0; ix < F->nkx; ++ix) {
                double kx = F->k0[0] * ix, ky = F->k0[1] * mode_of(iy, F->Ns[1]), kz = F->k0[2] * mode_of(iz, F->Ns[2]);
                if (kx * kx + ky * ky + kz * kz > kmax2)
                    for (int c = 0; c < 3; ++c) {
                        size_t u = uidx(F, c, ix, iy, iz);
                        F->uhat[2 * u] = F->uhat[2 * u + 1] = 0.0;
                    }
            }
}

/* Type-1 transform of (points, charges) into F->uhat with prefactor Gamma/V. */
static void lr_vorticity(const vpo_params* p, int64_t Nq, const double* points, const double* charges,
                         lr_field* F, vpo_stats* st) {
    double V = p->L[0] * p->L[1] * p->L[2];
    double pref = p->Gamma / V;
    size_t nu = (size_t)3 * F->Ns[2] * F->Ns[1] * F->nkx;
    memset(F->uhat, 0, sizeof(double) * 2 * nu);
    if (p->longrange_exact) {
        /* ExactSumBackend (exact_sum.jl:72-89): direct sums with separable phases */
#pragma omp parallel
        {
            int nmax = F->Ns[0] > F->Ns[1] ? F->Ns[0] : F->Ns[1];
            if (F->Ns[2] > nmax) nmax = F->Ns[2];
            cplx* ex = (cplx*)malloc(sizeof(cplx) * nmax);
            cplx* ey = (cplx*)malloc(sizeof(cplx) * nmax);
            cplx* ez = (cplx*)malloc(sizeof(cplx) * nmax);
#pragma omp for
            for (int iz = 0; iz < F->Ns[2]; ++iz) {
                for (int64_t j = 0; j < Nq; ++j) {
                    const double* X = points + 3 * j;
                    double kz = F->k0[2] * mode_of(iz, F->Ns[2]);
                    cplx pz = cexp(-I * kz * X[2]);
                    for (int ix = 0; ix < F->nkx; ++ix) ex[ix] = cexp(-I * F->k0[0] * ix * X[0]);
                    for (int iy = 0; iy < F->Ns[1]; ++iy) ey[iy] = cexp(-I * F->k0[1] * mode_of(iy, F->Ns[1]) * X[1]);
                    for (int iy = 0; iy < F->Ns[1]; ++iy) {
                        cplx pyz = pz * ey[iy];
                        for (int ix = 0; ix < F->nkx; ++ix) {
                            cplx ph = pyz * ex[ix];
                            for (int c = 0; c < 3; ++c) {
                                size_t u = uidx(F, c, ix, iy, iz);
                                double qv = pref * charges[3 * j + c];
                                F->uhat[2 * u] += qv * creal(ph);
                                F->uhat[2 * u + 1] += qv * cimag(ph);
                            }
                        }
                    }
                }
            }
            free(ex); free(ey); free(ez);
        }
        ensure_hermitian(F);
        return;
    }
    /* NUFFT type 1 with the ES kernel on the oversampled grid */
    int n[3], m = p->m;
    for (int d = 0; d < 3; ++d) n[d] = vpo_fft_size(F->Ns[d], p->sigma);
    double beta = es_beta(p);
    g_kernel_kind = p->nufft_kernel;
    if (st) { for (int d = 0; d < 3; ++d) st->fft_n[d] = n[d]; st->es_beta = beta; }
    size_t ng = (size_t)n[0] * n[1] * n[2];
    double* grid = (double*)calloc(3 * ng, sizeof(double));
    int w = 2 * m;
    /* z-block colouring so that threads never write the same grid plane */
    int nb = n[2] / w;
    if (nb % 2) nb--;
    if (nb < 2) nb = 1;
    for (int colour = 0; colour < (nb >= 2 ? 2 : 1); ++colour) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int b = colour; b < nb; b += (nb >= 2 ? 2 : 1)) {
            double phi[3][32];
            int i0[3];
            for (int64_t j = 0; j < Nq; ++j) {
                double xs[3];
                for (int d = 0; d < 3; ++d) xs[d] = points[3 * j + d] * (2.0 * VPO_PI / p->L[d]);
                double hz = 2.0 * VPO_PI / n[2];
                int zs = (int)floor(xs[2] / hz) - m + 1;
                int zr = (int)pmod(zs, n[2]);
                int blk = (int)((long)zr * nb / n[2]);
                if (blk != b) continue;
                for (int d = 0; d < 3; ++d) {
                    double h = 2.0 * VPO_PI / n[d];
                    double xh = xs[d] / h;
                    i0[d] = (int)floor(xh) - m + 1;
                    for (int s = 0; s < w; ++s) phi[d][s] = es_kernel(xh - (i0[d] + s), m, beta);
                }
                const double* qc = charges + 3 * j;
                for (int sz = 0; sz < w; ++sz) {
                    long iz = pmod(i0[2] + sz, n[2]);
                    for (int sy = 0; sy < w; ++sy) {
                        long iy = pmod(i0[1] + sy, n[1]);
                        double fyz = phi[2][sz] * phi[1][sy];
                        for (int sx = 0; sx < w; ++sx) {
                            long ix = pmod(i0[0] + sx, n[0]);
                            double f = fyz * phi[0][sx];
                            size_t g = ((size_t)iz * n[1] + iy) * n[0] + ix;
                            for (int c = 0; c < 3; ++c) grid[c * ng + g] += f * qc[c];
                        }
                    }
                }
            }
        }
    }
    /* forward FFT of each component and deconvolution onto the Ns modes */
    double* dec[3];
    for (int d = 0; d < 3; ++d) {
        dec[d] = (double*)malloc(sizeof(double) * F->Ns[d]);
        for (int i = 0; i < F->Ns[d]; ++i) {
            int k = (d == 0) ? i : mode_of(i, F->Ns[d]);
            if (d == 0 && i >= F->nkx) continue;
            dec[d][i] = 1.0 / es_hat(2.0 * VPO_PI * k / n[d], m, beta);
        }
    }
    cplx* cg = (cplx*)malloc(sizeof(cplx) * ng);
    for (int c = 0; c < 3; ++c) {
        for (size_t g = 0; g < ng; ++g) cg[g] = grid[c * ng + g];
        fft3(cg, n, -1);
        for (int iz = 0; iz < F->Ns[2]; ++iz)
            for (int iy = 0; iy < F->Ns[1]; ++iy)
                for (int ix = 0; ix < F->nkx; ++ix) {
                    long gz = pmod(mode_of(iz, F->Ns[2]), n[2]);
                    long gy = pmod(mode_of(iy, F->Ns[1]), n[1]);
                    cplx v = cg[(gz * n[1] + gy) * n[0] + ix] * (pref * dec[0][ix] * dec[1][iy] * dec[2][iz]);
                    size_t u = uidx(F, c, ix, iy, iz);
                    F->uhat[2 * u] = creal(v);
                    F->uhat[2 * u + 1] = cimag(v);
                }
    }
    free(cg);
    for (int d = 0; d < 3; ++d) free(dec[d]);
    free(grid);
    ensure_hermitian(F);
}

/* Apply the Fourier operator for `field` (0 = velocity, 1 = streamfunction) times the
 * Ewald Gaussian, and interpolate to the nodes (type 2). */
static void lr_interpolate(const vpo_params* p, const lr_field* W, int field, int64_t Np,
                           const double* nodes_f, double* out) {
    int Ns0 = W->Ns[0], Ns1 = W->Ns[1], Ns2 = W->Ns[2], nkx = W->nkx;
    size_t nu = (size_t)Ns2 * Ns1 * nkx;
    /* û of the requested field, smoothed by exp(-k^2/4 alpha^2) (Gaussian) or by the
     * Kaiser-Bessel filter */
    cplx* u = (cplx*)malloc(sizeof(cplx) * 3 * nu);
    double beta_g = -1.0 / (4.0 * p->alpha * p->alpha);
    for (int iz = 0; iz < Ns2; ++iz)
        for (int iy = 0; iy < Ns1; ++iy)
            for (int ix = 0; ix < nkx; ++ix) {
                double k[3] = {W->k0[0] * ix, W->k0[1] * mode_of(iy, Ns1), W->k0[2] * mode_of(iz, Ns2)};
                double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                double k2inv = (k2 == 0.0) ? 0.0 : 1.0 / k2;
                double E = p->splitting == 1 ? kb_fourier(p->kb_beta, p->rcut, k2) : exp(beta_g * k2);
                cplx w[3];
                for (int c = 0; c < 3; ++c) {
                    size_t q = uidx(W, c, ix, iy, iz);
                    w[c] = W->uhat[2 * q] + I * W->uhat[2 * q + 1];
                }
                cplx r[3];
                if (field == 1) {
                    for (int c = 0; c < 3; ++c) r[c] = w[c] * k2inv;
                } else {
                    /* i k x w / k^2 */
                    cplx iw[3] = {I * w[0], I * w[1], I * w[2]};
                    r[0] = (k[1] * iw[2] - k[2] * iw[1]) * k2inv;
                    r[1] = (k[2] * iw[0] - k[0] * iw[2]) * k2inv;
                    r[2] = (k[0] * iw[1] - k[1] * iw[0]) * k2inv;
                }
                size_t base = ((size_t)iz * Ns1 + iy) * nkx + ix;
                for (int c = 0; c < 3; ++c) u[c * nu + base] = r[c] * E;
            }
    if (p->longrange_exact) {
        /* exact_sum.jl:91-121 */
#pragma omp parallel for schedule(dynamic, 4)
        for (int64_t i = 0; i < Np; ++i) {
            const double* X = nodes_f + 3 * i;
            cplx ex[1024], ey[1024];
            for (int ix = 0; ix < nkx; ++ix) ex[ix] = cexp(I * W->k0[0] * ix * X[0]);
            for (int iy = 0; iy < Ns1; ++iy) ey[iy] = cexp(I * W->k0[1] * mode_of(iy, Ns1) * X[1]);
            double acc[3] = {0, 0, 0};
            for (int iz = 0; iz < Ns2; ++iz) {
                cplx pz = cexp(I * W->k0[2] * mode_of(iz, Ns2) * X[2]);
                for (int iy = 0; iy < Ns1; ++iy) {
                    cplx pyz = pz * ey[iy];
                    for (int ix = 0; ix < nkx; ++ix) {
                        cplx z = pyz * ex[ix];
                        double fac = (ix == 0 || ix == nkx - 1) ? 1.0 : 2.0;
                        size_t base = ((size_t)iz * Ns1 + iy) * nkx + ix;
                        for (int c = 0; c < 3; ++c) acc[c] += fac * creal(u[c * nu + base] * z);
                    }
                }
            }
            for (int c = 0; c < 3; ++c) out[3 * i + c] = acc[c];
        }
        (void)Ns0;
        free(u);
        return;
    }
    int n[3], m = p->m, w = 2 * m;
    for (int d = 0; d < 3; ++d) n[d] = vpo_fft_size(W->Ns[d], p->sigma);
    double beta = es_beta(p);
    g_kernel_kind = p->nufft_kernel;
    double* dec[3];
    for (int d = 0; d < 3; ++d) {
        dec[d] = (double*)malloc(sizeof(double) * W->Ns[d]);
        for (int i = 0; i < W->Ns[d]; ++i) {
            if (d == 0 && i >= nkx) continue;
            int k = (d == 0) ? i : mode_of(i, W->Ns[d]);
            dec[d][i] = 1.0 / es_hat(2.0 * VPO_PI * k / n[d], m, beta);
        }
    }
    size_t ng = (size_t)n[0] * n[1] * n[2];
    double* grid = (double*)malloc(sizeof(double) * 3 * ng);
    cplx* cg = (cplx*)malloc(sizeof(cplx) * ng);
    for (int c = 0; c < 3; ++c) {
        memset(cg, 0, sizeof(cplx) * ng);
        for (int iz = 0; iz < Ns2; ++iz)
            for (int iy = 0; iy < Ns1; ++iy)
                for (int ix = 0; ix < nkx; ++ix) {
                    size_t base = ((size_t)iz * Ns1 + iy) * nkx + ix;
                    cplx v = u[c * nu + base] * (dec[0][ix] * dec[1][iy] * dec[2][iz]);
                    long gz = pmod(mode_of(iz, Ns2), n[2]), gy = pmod(mode_of(iy, Ns1), n[1]);
                    cg[(gz * n[1] + gy) * n[0] + ix] += v;
                    if (ix > 0) {
                        long gz2 = pmod(-mode_of(iz, Ns2), n[2]), gy2 = pmod(-mode_of(iy, Ns1), n[1]);
                        cg[(gz2 * n[1] + gy2) * n[0] + (n[0] - ix)] += conj(v);
                    }
                }
        fft3(cg, n, +1);
        for (size_t g = 0; g < ng; ++g) grid[c * ng + g] = creal(cg[g]);
    }
    free(cg);
#pragma omp parallel for
    for (int64_t i = 0; i < Np; ++i) {
        double phi[3][32];
        int i0[3];
        for (int d = 0; d < 3; ++d) {
            double h = 2.0 * VPO_PI / n[d];
            double xh = nodes_f[3 * i + d] * (2.0 * VPO_PI / p->L[d]) / h;
            i0[d] = (int)floor(xh) - m + 1;
            for (int s = 0; s < w; ++s) phi[d][s] = es_kernel(xh - (i0[d] + s), m, beta);
        }
        double acc[3] = {0, 0, 0};
        for (int sz = 0; sz < w; ++sz) {
            long iz = pmod(i0[2] + sz, n[2]);
            for (int sy = 0; sy < w; ++sy) {
                long iy = pmod(i0[1] + sy, n[1]);
                double fyz = phi[2][sz] * phi[1][sy];
                for (int sx = 0; sx < w; ++sx) {
                    long ix = pmod(i0[0] + sx, n[0]);
                    double f = fyz * phi[0][sx];
                    size_t g = ((size_t)iz * n[1] + iy) * n[0] + ix;
                    for (int c = 0; c < 3; ++c) acc[c] += f * grid[c * ng + g];
                }
            }
        }
        for (int c = 0; c < 3; ++c) out[3 * i + c] = acc[c];
    }
    for (int d = 0; d < 3; ++d) free(dec[d]);
    free(grid);
    free(u);
}

static void lr_field_init(const vpo_params* p, lr_field* F) {
    for (int d = 0; d < 3; ++d) {
        F->Ns[d] = p->Ns[d];
        F->k0[d] = 2.0 * VPO_PI / p->L[d];
    }
    F->nkx = p->Ns[0] / 2 + 1;
    F->uhat = (double*)calloc((size_t)2 * 3 * F->Ns[2] * F->Ns[1] * F->nkx, sizeof(double));
}

int vpo_vorticity_fourier(const vpo_params* p, int64_t Nq, const double* points, const double* charges,
                          double* uhat_out, vpo_stats* st) {
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
    if (is_open(p) || !ewald_on(p)) return -1;
    lr_field F;
    lr_field_init(p, &F);
    lr_vorticity(p, Nq, points, charges, &F, st);
    if (p->truncate_spherical) truncate_spherical(p, &F);
    memcpy(uhat_out, F.uhat, sizeof(double) * 2 * 3 * F.Ns[2] * F.Ns[1] * F.nkx);
    free(F.uhat);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* compute_on_nodes!  (reference: src/BiotSavart/BiotSavart.jl:395-612)      */
/* ------------------------------------------------------------------------- */

/* Streamfunction factor of a uniform background vorticity (background_vorticity_correction_factor):
 * 1 / (4 alpha^2) for the Gaussian splitting (gaussian.jl:241), and for the Kaiser-Bessel one
 * C = int_0^rcut r^2 f(r) dr / 2 with f(r) = beta / (rcut sinh beta) I0(beta sqrt(1 - r^2/rcut^2))
 * (kaiser_bessel.jl:160-165, 280), here by 64-point Gauss-Legendre quadrature (the integrand is
 * analytic in r^2 on [0, rcut]). */
double vpo_background_factor(const vpo_params* p) {
    if (p->splitting == 1) {
        double z[64], w[64];
        vpo_gl_rule(64, z, w);
        const double rc = p->rcut, beta = p->kb_beta;
        double acc = 0.0;
        for (int q = 0; q < 64; ++q) {
            const double r = z[q] * rc, u = r / rc;
            const double f = beta / (rc * sinh(beta)) * bessel_i0(beta * sqrt(fmax(0.0, 1.0 - u * u)));
            acc += w[q] * rc * r * r * f;
        }
        return acc / 2.0;
    }
    return 1.0 / (4.0 * p->alpha * p->alpha);
}

/* background_vorticity_correction! (BiotSavart.jl:255-286): with a non-zero sum p of the
 * end-to-end offsets, psi += -(p Gamma / V) C on every node. */
static void background_correction(const vpo_params* p, int nfil, int64_t Np, double* psi) {
    if (!p->fil_offsets || !psi) return;
    double ptot[3] = {0, 0, 0};
    for (int f = 0; f < nfil; ++f)
        for (int d = 0; d < 3; ++d) ptot[d] += p->fil_offsets[3 * f + d];
    /* isapprox(p + Ls, Ls) with the default rtol sqrt(eps): nothing to do */
    double dn = 0.0, na = 0.0, nb = 0.0;
    for (int d = 0; d < 3; ++d) {
        dn += ptot[d] * ptot[d];
        na += (ptot[d] + p->L[d]) * (ptot[d] + p->L[d]);
        nb += p->L[d] * p->L[d];
    }
    if (sqrt(dn) <= sqrt(2.220446049250313e-16) * fmax(sqrt(na), sqrt(nb))) return;
    const double V = p->L[0] * p->L[1] * p->L[2];
    const double C = vpo_background_factor(p);
    double back[3];
    for (int d = 0; d < 3; ++d) back[d] = -ptot[d] * (p->Gamma / V) * C;
    for (int64_t i = 0; i < Np; ++i)
        for (int d = 0; d < 3; ++d) psi[3 * i + d] += back[d];
}

int vpo_compute_on_nodes(const vpo_params* p, int nfil, const int64_t* offsets, const double* nodes_xyz,
                         int lia_mode, int shortrange, int longrange,
                         double* vel_out, double* psi_out, vpo_stats* st) {
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
    if (!vel_out && !psi_out) return -1;
    int64_t Np = offsets[nfil];
    int nq = p->nquad;
    int64_t Nq = Np * nq;
    if (st) memset(st, 0, sizeof *st);
    if (p->splitting == 1) {
        kb_free(&g_kb);
        if (!(p->kb_beta > 0) || !(p->rcut > 0) || kb_build(p->kb_beta, p->rcut, p->kb_rtol, &g_kb)) return -3;
    }
    if (ewald_on(p)) {
        for (int d = 0; d < 3; ++d)
            if (!(p->L[d] > 0) || 2.0 * p->rcut > p->L[d]) return -3;
        if (p->nsubdiv > 0)
            for (int d = 0; d < 3; ++d)
                if (p->rcut > (double)p->nsubdiv / (2.0 * p->nsubdiv + 1.0) * p->L[d]) return -3;
    }
    double* nodes_f = (double*)malloc(sizeof(double) * 3 * Np);
    int32_t* idx_prev = (int32_t*)malloc(sizeof(int32_t) * Np);
    double* d1 = (double*)malloc(sizeof(double) * 3 * Np);
    double* d2 = (double*)malloc(sizeof(double) * 3 * Np);
    double* dm = (double*)malloc(sizeof(double) * Np);
    double* dp = (double*)malloc(sizeof(double) * Np);
    double* points = (double*)malloc(sizeof(double) * 3 * Nq);
    double* charges = (double*)malloc(sizeof(double) * 3 * Nq);
    int err = vpo_point_data(p, nfil, offsets, nodes_xyz, nodes_f, idx_prev, d1, d2, dm, dp, points, charges);
    if (err) goto done;
    if (vel_out) memset(vel_out, 0, sizeof(double) * 3 * Np);
    if (psi_out) memset(psi_out, 0, sizeof(double) * 3 * Np);

    int with_long = longrange && lia_mode != 2 && ewald_on(p);
    if (with_long) {
        lr_field F;
        lr_field_init(p, &F);
        lr_vorticity(p, Nq, points, charges, &F, st);
        if (p->truncate_spherical) truncate_spherical(p, &F);
        double* tmp = (double*)malloc(sizeof(double) * 3 * Np);
        if (psi_out) {
            lr_interpolate(p, &F, 1, Np, nodes_f, tmp);
            for (int64_t i = 0; i < 3 * Np; ++i) psi_out[i] += tmp[i];
        }
        if (vel_out) {
            lr_interpolate(p, &F, 0, Np, nodes_f, tmp);
            for (int64_t i = 0; i < 3 * Np; ++i) vel_out[i] += tmp[i];
        }
        free(tmp);
        free(F.uhat);
    }
    if (shortrange) {
        double* sv = vel_out ? (double*)calloc(3 * Np, sizeof(double)) : NULL;
        double* sp = psi_out ? (double*)calloc(3 * Np, sizeof(double)) : NULL;
        if (lia_mode == 1 || lia_mode == 2) local_term(p, Np, d1, d2, dm, dp, sv, sp);
        if (lia_mode != 2) {
            pairs(p, Np, Nq, nodes_f, idx_prev, points, charges, sv, sp, st);
            remove_self(p, Np, nodes_f, idx_prev, points, charges, sv, sp);
        }
        for (int64_t i = 0; i < 3 * Np; ++i) {
            if (sv) vel_out[i] += sv[i];
            if (sp) psi_out[i] += sp[i];
        }
        free(sv);
        free(sp);
        if (lia_mode != 2 && p->lia_segment_fraction > 0) {
            for (int f = 0; f < nfil; ++f) {
                spline_t S;
                int64_t off = offsets[f];
                if (spline_build(&S, (int)(offsets[f + 1] - off), nodes_xyz + 3 * off,
                                 p->fil_offsets ? p->fil_offsets + 3 * f : NULL) != 0) {
                    err = -2;
                    break;
                }
                local_integrals(p, &S, off, nodes_f, vel_out, psi_out);
                spline_free(&S);
            }
        }
        if (lia_mode != 2 && ewald_on(p)) background_correction(p, nfil, Np, psi_out);
    }
done:
    free(nodes_f); free(idx_prev); free(d1); free(d2); free(dm); free(dp); free(points); free(charges);
    return err;
}
