// Filament geometry on the device: chordal knots, periodic quintic spline interpolation and
// the point data of add_point_charges! (src/BiotSavart/pointdata_impl.jl:41-108).
//
// One warp per filament solves the cyclic pentadiagonal B-spline collocation system
// (src/Filaments/spline/quintic.jl:9-100 solves the same system): the band part is
// factorised by elimination without pivoting (collocation matrices of B-splines are totally
// positive), the seven right-hand sides (x, y, z and the four wrap-around columns) are swept
// by seven lanes in parallel, and the corners are folded back with the Woodbury identity.
// A second kernel evaluates the splines at the nodes and quadrature points, one thread per node.
#include "vpbs_internal.cuh"
#include "periodic.cuh"

namespace vpbs {
namespace {

struct FilView {
    const double* t;  // knots of this filament (n values, t[0] = 0)
    double T;         // knot period
    int n;
    double o[3];      // end-to-end offset (zero for a closed filament)
};

// FilView of filament fidx; `foff` ([nfil][3] end-to-end offsets) may be null (closed filaments).
__device__ __forceinline__ FilView fil_view(const double* knots, const double* periods, const double* foff,
                                            int64_t off, int n, int64_t fidx) {
    FilView f{knots + off, periods[fidx], n, {0.0, 0.0, 0.0}};
    if (foff) {
        f.o[0] = foff[3 * fidx];
        f.o[1] = foff[3 * fidx + 1];
        f.o[2] = foff[3 * fidx + 2];
    }
    return f;
}

// j mod n in [0, n).  The spline code only asks for j in [-n, 2n) (n >= 5 nodes, indices at most 6
// away from a node), which takes no division; other j take the general form.
__device__ __forceinline__ long pmodl(long j, long n) {
    if (j >= 0 && j < n) return j;
    if (j < 0 && j >= -n) return j + n;
    if (j >= n && j < 2 * n) return j - n;
    long r = j % n;
    return r < 0 ? r + n : r;
}

// Knot t_j of the periodically extended sequence, t_{j + q n} = t_j + q T (the same rounding as
// t[j - q n] + q T for every q: q = +-1 adds or subtracts T exactly as the general form does).
__device__ __forceinline__ double knot_at(const FilView& f, long j) {
    const long n = f.n;
    if (j >= 0 && j < n) return f.t[j];
    if (j < 0 && j >= -n) return f.t[j + n] - f.T;
    if (j >= n && j < 2 * n) return f.t[j - n] + f.T;
    long q = (j >= 0) ? j / n : -((-j + n - 1) / n);
    return f.t[j - q * n] + (double)q * f.T;
}

// de Boor's BSPLVB: N[s] = B_{i-K+1+s, K}(x) for x in [t_i, t_{i+1}).
template <int K>
__device__ __forceinline__ void bsplvb(const FilView& f, long i, double x, double (&N)[K]) {
    double left[K], right[K];
    N[0] = 1.0;
#pragma unroll
    for (int r = 1; r < K; ++r) {
        left[r] = x - knot_at(f, i + 1 - r);
        right[r] = knot_at(f, i + r) - x;
        double saved = 0.0;
#pragma unroll
        for (int s = 0; s < r; ++s) {
            double tmp = N[s] / (right[s + 1] + left[r - s]);
            N[s] = saved + right[s + 1] * tmp;
            saved = left[r - s] * tmp;
        }
        N[r] = saved;
    }
}

// Spline derivative `D` (0, 1, 2) at local coordinate zeta on segment i.
// coef: AoS [n][3] coefficients of order 6 - D for this filament.
template <int D>
__device__ __forceinline__ void eval_seg(const FilView& f, const double* coef, long i, double zeta, double out[3]) {
    constexpr int K = 6 - D;
    double ti = knot_at(f, i), ti1 = knot_at(f, i + 1);
    double x = (1.0 - zeta) * ti + zeta * ti1;
    double N[K];
    bsplvb<K>(f, i, x, N);
    out[0] = out[1] = out[2] = 0.0;
#pragma unroll
    for (int s = 0; s < K; ++s) {
        long j = pmodl(i - K + 1 + s, f.n);
        out[0] += coef[3 * j + 0] * N[s];
        out[1] += coef[3 * j + 1] * N[s];
        out[2] += coef[3 * j + 2] * N[s];
    }
    // an unclosed (infinite) filament is the periodic spline y plus (x / T) offset (spline.jl:185-194)
    if (D == 0) {
        const double r = x / f.T;
#pragma unroll
        for (int d = 0; d < 3; ++d) out[d] += r * f.o[d];
    } else if (D == 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) out[d] += f.o[d] / f.T;
    }
}

// Knots t_{i-4} .. t_{i+5} around segment i and the reciprocals of the knot spans the B-spline
// recurrence divides by, 1 / (t_{i+s+1} - t_{i+s+1-r}) for r = 1..5 and s < r (spline.jl:116-160 uses
// the same recurrence): the spans do not depend on the evaluation point, so every evaluation on the
// segment shares one division per span.
struct SegBasis {
    double t[10];    // t[4 + j] = t_{i+j}
    double inv[15];  // inv[r (r - 1) / 2 + s]
};

__device__ __forceinline__ void seg_basis_init(const FilView& f, long i, SegBasis& B) {
#pragma unroll
    for (int j = -4; j <= 5; ++j) B.t[4 + j] = knot_at(f, i + j);
#pragma unroll
    for (int r = 1; r <= 5; ++r)
#pragma unroll
        for (int s = 0; s < r; ++s) B.inv[r * (r - 1) / 2 + s] = 1.0 / (B.t[5 + s] - B.t[5 + s - r]);
}

// bsplvb<K> on the segment of B: N[s] = B_{i-K+1+s, K}(x) for x in [t_i, t_{i+1}).
template <int K>
__device__ __forceinline__ void bsplvb_seg(const SegBasis& B, double x, double (&N)[K]) {
    double left[K], right[K];
    N[0] = 1.0;
#pragma unroll
    for (int r = 1; r < K; ++r) {
        left[r] = x - B.t[5 - r];
        right[r] = B.t[4 + r] - x;
        double saved = 0.0;
#pragma unroll
        for (int s = 0; s < r; ++s) {
            const double tmp = N[s] * B.inv[r * (r - 1) / 2 + s];
            N[s] = saved + right[s + 1] * tmp;
            saved = left[r - s] * tmp;
        }
        N[r] = saved;
    }
}

// eval_seg<D> with the segment's shared knots and spans.
template <int D>
__device__ __forceinline__ void eval_seg_b(const FilView& f, const SegBasis& B, const double* coef, long i,
                                           double zeta, double out[3]) {
    constexpr int K = 6 - D;
    const double x = (1.0 - zeta) * B.t[4] + zeta * B.t[5];
    double N[K];
    bsplvb_seg<K>(B, x, N);
    out[0] = out[1] = out[2] = 0.0;
#pragma unroll
    for (int s = 0; s < K; ++s) {
        const long j = pmodl(i - K + 1 + s, f.n);
        out[0] += coef[3 * j + 0] * N[s];
        out[1] += coef[3 * j + 1] * N[s];
        out[2] += coef[3 * j + 2] * N[s];
    }
    if (D == 0) {
        const double r = x / f.T;
#pragma unroll
        for (int d = 0; d < 3; ++d) out[d] += r * f.o[d];
    } else if (D == 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) out[d] += f.o[d] / f.T;
    }
}

// Solve the 4x4 Woodbury capacitance system with partial pivoting (3 right-hand sides).
__device__ void solve4(double H[4][4], double r[4][3]) {
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int i = c + 1; i < 4; ++i)
            if (fabs(H[i][c]) > fabs(H[piv][c])) piv = i;
        if (piv != c) {
            for (int j = 0; j < 4; ++j) { double t = H[c][j]; H[c][j] = H[piv][j]; H[piv][j] = t; }
            for (int j = 0; j < 3; ++j) { double t = r[c][j]; r[c][j] = r[piv][j]; r[piv][j] = t; }
        }
        for (int i = c + 1; i < 4; ++i) {
            double fct = H[i][c] / H[c][c];
            for (int j = c; j < 4; ++j) H[i][j] -= fct * H[c][j];
            for (int j = 0; j < 3; ++j) r[i][j] -= fct * r[c][j];
        }
    }
    for (int c = 3; c >= 0; --c)
        for (int j = 0; j < 3; ++j) {
            double s = r[c][j];
            for (int k = c + 1; k < 4; ++k) s -= H[c][k] * r[k][j];
            r[c][j] = s / H[c][c];
        }
}

// One warp per filament.  Work space: 12 doubles per node (5 band + 7 right-hand sides), in
// dynamic shared memory (smem_n doubles x 12 per warp) when smem_n > 0, else in `scratch`.
// keep_knots: reuse the knots and periods already in `knots` / `periods` (the knots frozen
// inside a time step, RK4.jl with update_coefficients!(f; knots = ts_base)).
__global__ void __launch_bounds__(128) spline_solve_kernel(
    int64_t nfil, const int64_t* __restrict__ offsets, const double* __restrict__ X,
    double* __restrict__ knots, double* __restrict__ periods, int32_t* __restrict__ fil_of_node,
    double* __restrict__ coef, double* __restrict__ dcoef1, double* __restrict__ dcoef2,
    double* __restrict__ scratch, int32_t* __restrict__ status, int smem_n, int keep_knots,
    const double* __restrict__ foff) {
    extern __shared__ double sm_work[];
    const int lane = threadIdx.x & 31;
    const int64_t fidx = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (fidx >= nfil) return;
    const int64_t off = offsets[fidx];
    const int n = (int)(offsets[fidx + 1] - off);
    if (n < 5 || (smem_n > 0 && n > smem_n)) {
        if (lane == 0) atomicExch(status, 1);
        return;
    }
    const double* Xf = X + 3 * off;
    double* t = knots + off;
    double* band = smem_n > 0 ? sm_work + (size_t)(threadIdx.x >> 5) * 12 * smem_n : scratch + 12 * off;  // [n][5]
    double* Y = band + 5 * (int64_t)n;      // [n][7]
    double* c = coef + 3 * off;
    double* c1 = dcoef1 + 3 * off;
    double* c2 = dcoef2 + 3 * off;

    // 1. chordal knots: warp-wide inclusive scan of segment lengths (parametrisations.jl:43-44)
    double carry = keep_knots ? periods[fidx] : 0.0;
    for (int base = 0; base < n && !keep_knots; base += 32) {
        int i = base + lane;
        double len = 0.0;
        if (i < n) {
            int j = (i + 1 == n) ? 0 : i + 1;
            double dx = Xf[3 * j] - Xf[3 * i], dy = Xf[3 * j + 1] - Xf[3 * i + 1], dz = Xf[3 * j + 2] - Xf[3 * i + 2];
            if (j == 0 && foff) {  // closing segment of an unclosed filament: to X_0 + offset
                dx += foff[3 * fidx];
                dy += foff[3 * fidx + 1];
                dz += foff[3 * fidx + 2];
            }
            len = sqrt(dx * dx + dy * dy + dz * dz);
            fil_of_node[off + i] = (int32_t)fidx;
        }
        double incl = len;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
            double v = __shfl_up_sync(0xffffffffu, incl, s);
            if (lane >= s) incl += v;
        }
        if (i < n) t[i] = carry + (incl - len);  // exclusive prefix: t_i
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    const double T = carry;
    if (lane == 0 && !keep_knots) periods[fidx] = T;
    __syncwarp();
    FilView f{t, T, n, {0.0, 0.0, 0.0}};
    // an unclosed filament is interpolated as the periodic y_i = X_i - (t_i / T) offset
    // (spline.jl:163-182, quintic.jl:9-17)
    const double o0 = foff ? foff[3 * fidx] : 0.0, o1 = foff ? foff[3 * fidx + 1] : 0.0,
                 o2 = foff ? foff[3 * fidx + 2] : 0.0;

    // 2. collocation rows, band part only (corners handled below)
    for (int i = lane; i < n; i += 32) {
        double N[6];
        bsplvb<6>(f, i, knot_at(f, i), N);
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            int col = i + s - 2;
            band[5 * i + s] = (col >= 0 && col < n) ? N[s] : 0.0;
        }
        const double r = t[i] / T;
        Y[7 * i + 0] = Xf[3 * i + 0] - r * o0;
        Y[7 * i + 1] = Xf[3 * i + 1] - r * o1;
        Y[7 * i + 2] = Xf[3 * i + 2] - r * o2;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int ur = (q == 0) ? 0 : (q == 1) ? 1 : (q == 2) ? n - 2 : n - 1;
            Y[7 * i + 3 + q] = (i == ur) ? 1.0 : 0.0;
        }
    }
    __syncwarp();

    // 3. pentadiagonal LU without pivoting (serial, lane 0), as a register recurrence: row i of
    //    the band (e, d, c, b, a at columns i-2..i+2) becomes (l2, l1, 1/u0, u1, u2):
    //    l2 = e/u0[i-2], l1 = (d - l2 u1[i-2])/u0[i-1], u0 = c - l2 u2[i-2] - l1 u1[i-1],
    //    u1 = b - l1 u2[i-1], u2 = a.
    if (lane == 0) {
        double iu0_m2 = 0.0, u1_m2 = 0.0, u2_m2 = 0.0;  // row i-2
        double iu0_m1 = 0.0, u1_m1 = 0.0, u2_m1 = 0.0;  // row i-1
        for (int i = 0; i < n; ++i) {
            double* r = band + 5 * i;
            const double e = r[0], d = r[1], c = r[2], b = r[3], a = r[4];
            const double l2 = e * iu0_m2;
            const double l1 = (d - l2 * u1_m2) * iu0_m1;
            const double u0 = c - l2 * u2_m2 - l1 * u1_m1;
            const double u1 = b - l1 * u2_m1;
            const double iu0 = 1.0 / u0;
            r[0] = l2;
            r[1] = l1;
            r[2] = iu0;
            r[3] = u1;
            r[4] = a;
            iu0_m2 = iu0_m1; u1_m2 = u1_m1; u2_m2 = u2_m1;
            iu0_m1 = iu0; u1_m1 = u1; u2_m1 = a;
        }
    }
    __syncwarp();

    // 4. forward / backward sweeps, one right-hand side per lane (register recurrences)
    if (lane < 7) {
        const int q = lane;
        double z1 = 0.0, z2 = 0.0;  // z[i-1], z[i-2]
        for (int i = 0; i < n; ++i) {
            const double* r = band + 5 * i;
            const double z = Y[7 * i + q] - r[1] * z1 - r[0] * z2;
            Y[7 * i + q] = z;
            z2 = z1;
            z1 = z;
        }
        double x1 = 0.0, x2 = 0.0;  // x[i+1], x[i+2]
        for (int i = n - 1; i >= 0; --i) {
            const double* r = band + 5 * i;
            const double x = (Y[7 * i + q] - r[3] * x1 - r[4] * x2) * r[2];
            Y[7 * i + q] = x;
            x2 = x1;
            x1 = x;
        }
    }
    __syncwarp();

    // 5. Woodbury correction: corners W of rows 0, 1, n-2, n-1
    __shared__ double sh_s[4][4][3];
    double (*s4)[3] = sh_s[threadIdx.x >> 5];
    if (lane == 0) {
        double H[4][4], rh[4][3];
        const int rows[4] = {0, 1, n - 2, n - 1};
        for (int r = 0; r < 4; ++r) {
            for (int q = 0; q < 4; ++q) H[r][q] = (r == q) ? 1.0 : 0.0;
            for (int d = 0; d < 3; ++d) rh[r][d] = 0.0;
            int i = rows[r];
            double N[6];
            bsplvb<6>(f, i, knot_at(f, i), N);
            for (int s = 0; s < 5; ++s) {
                int col = i + s - 2;
                if (col >= 0 && col < n) continue;
                int cw = (int)pmodl(col, n);
                for (int q = 0; q < 4; ++q) H[r][q] += N[s] * Y[7 * cw + 3 + q];
                for (int d = 0; d < 3; ++d) rh[r][d] += N[s] * Y[7 * cw + d];
            }
        }
        solve4(H, rh);
        for (int r = 0; r < 4; ++r)
            for (int d = 0; d < 3; ++d) s4[r][d] = rh[r][d];
    }
    __syncwarp();

    // 6. coefficients c_j = u_{j+3}, u = y - Z s
    for (int i = lane; i < n; i += 32) {
        int j = (int)pmodl(i - 3, n);  // u_i = c_{i-3}
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double u = Y[7 * i + d];
#pragma unroll
            for (int q = 0; q < 4; ++q) u -= Y[7 * i + 3 + q] * s4[q][d];
            c[3 * j + d] = u;
        }
    }
    __syncwarp();
    // 7. derivative coefficients (spline derivative recurrence, spline.jl:301-319)
    for (int j = lane; j < n; j += 32) {
        int jm = (j == 0) ? n - 1 : j - 1;
        double den = knot_at(f, j + 5) - knot_at(f, j);
#pragma unroll
        for (int d = 0; d < 3; ++d) c1[3 * j + d] = 5.0 * (c[3 * j + d] - c[3 * jm + d]) / den;
    }
    __syncwarp();
    for (int j = lane; j < n; j += 32) {
        int jm = (j == 0) ? n - 1 : j - 1;
        double den = knot_at(f, j + 4) - knot_at(f, j);
#pragma unroll
        for (int d = 0; d < 3; ++d) c2[3 * j + d] = 4.0 * (c1[3 * j + d] - c1[3 * jm + d]) / den;
    }
}

__device__ double seg_len(const FilView& f, const double* c1, long i, int nq, const double* qz, const double* qw,
                          double a, double b) {
    double dt = knot_at(f, i + 1) - knot_at(f, i);
    double acc = 0.0;
    for (int q = 0; q < nq; ++q) {
        double d[3];
        eval_seg<1>(f, c1, i, a + (b - a) * qz[q], d);
        acc += qw[q] * sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
    return dt * (b - a) * acc;
}

// One thread per node: point data of pointdata_impl.jl:65-108 and, when
// lia_segment_fraction is set, the local integrals of local_integrals.jl:253-293.
// FUSE: full segments without lia_segment_fraction (quadrature points written here); compiled
// separately so that the common path carries none of the other path's code.
template <bool FUSE>
__global__ void __launch_bounds__(128, FUSE ? 4 : 1) point_data_kernel(
    KParams K, int64_t Np, const int64_t* __restrict__ offsets, const int32_t* __restrict__ fil_of_node,
    const double* __restrict__ X, const double* __restrict__ knots, const double* __restrict__ periods,
    const double* __restrict__ coef, const double* __restrict__ dcoef1, const double* __restrict__ dcoef2,
    double* __restrict__ nodes, int32_t* __restrict__ idx_prev, double* __restrict__ d1, double* __restrict__ d2,
    double* __restrict__ dm, double* __restrict__ dp, double* __restrict__ points, double* __restrict__ charges,
    double* __restrict__ li_vel, double* __restrict__ li_psi, int want_li, int fuse_quad,
    const double* __restrict__ foff) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Np) return;
    const int fidx = fil_of_node[k];
    const int64_t off = offsets[fidx];
    const int n = (int)(offsets[fidx + 1] - off);
    const int i = (int)(k - off);
    const FilView f = fil_view(knots, periods, foff, off, n, fidx);
    const double* c = coef + 3 * off;
    const double* c1 = dcoef1 + 3 * off;
    const double* c2 = dcoef2 + 3 * off;
    const int64_t Nq = Np * K.nquad;

    double xf[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        xf[d] = fold(X[3 * k + d], K.L[d], K.open_domain);
        nodes[d * Np + k] = xf[d];
    }
    idx_prev[k] = (int32_t)(i == 0 ? off + n - 1 : k - 1);
    SegBasis B;
    seg_basis_init(f, i, B);
    double s1[3], s2[3];
    eval_seg_b<1>(f, B, c1, i, 0.0, s1);
    eval_seg_b<2>(f, B, c2, i, 0.0, s2);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        d1[d * Np + k] = s1[d];
        d2[d * Np + k] = s2[d];
    }
    const double g = K.lia_fraction;
    const bool has_g = g > 0;
    if (FUSE) {
        // full segments (no lia_segment_fraction): the quadrature points and charges of segment i
        // (as quad_points_kernel computes them) and its length from the same s' values, in the
        // operation order of seg_len; delta^- is the previous node's delta^+ (dm_from_prev_kernel)
        const double dt = B.t[5] - B.t[4];
        double acc = 0.0;
        for (int q = 0; q < K.nquad; ++q) {
            double s[3], sp[3];
            eval_seg_b<0>(f, B, c, i, K.qz[q], s);
            eval_seg_b<1>(f, B, c1, i, K.qz[q], sp);
            const int64_t mq = k * K.nquad + q;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                points[d * Nq + mq] = fold(s[d], K.L[d], K.open_domain);
                charges[d * Nq + mq] = K.qw[q] * dt * sp[d];
            }
            acc += K.qw[q] * sqrt(sp[0] * sp[0] + sp[1] * sp[1] + sp[2] * sp[2]);
        }
        dp[k] = dt * 1.0 * acc;
    } else {
        dm[k] = seg_len(f, c1, i - 1, K.nquad, K.qz, K.qw, has_g ? 1.0 - g : 0.0, 1.0);
        dp[k] = seg_len(f, c1, i, K.nquad, K.qz, K.qw, 0.0, has_g ? g : 1.0);
    }
    if (!FUSE && want_li) {
        // nonlia_integration_limits: ((0, 1-g), (g, 1))  (local_integrals.jl:103-104)
        double v[3] = {0, 0, 0}, ps[3] = {0, 0, 0};
        for (int side = 0; side < 2; ++side) {
            const long seg = side == 0 ? i - 1 : i;
            const double a = side == 0 ? 0.0 : g, b = side == 0 ? 1.0 - g : 1.0;
            const double dts = (knot_at(f, seg + 1) - knot_at(f, seg)) * (b - a);
            for (int q = 0; q < K.nquad_near; ++q) {
                const double y = a + (b - a) * K.qnz[q];
                double s[3], sp[3], r[3], qc[3];
                eval_seg<0>(f, c, seg, y, s);
                eval_seg<1>(f, c1, seg, y, sp);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    qc[d] = K.qnw[q] * dts * sp[d];
                    r[d] = deper(xf[d] - fold(s[d], K.L[d], K.open_domain), K.L[d], K.Lh[d], K.open_domain);
                }
                const double rinv = 1.0 / sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                const double r3 = rinv * rinv * rinv;
                v[0] += r3 * (qc[1] * r[2] - qc[2] * r[1]);
                v[1] += r3 * (qc[2] * r[0] - qc[0] * r[2]);
                v[2] += r3 * (qc[0] * r[1] - qc[1] * r[0]);
#pragma unroll
                for (int d = 0; d < 3; ++d) ps[d] += rinv * qc[d];
            }
        }
        const double pref = K.Gamma / (4.0 * kPi);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            li_vel[d * Np + k] = pref * v[d];
            li_psi[d * Np + k] = pref * ps[d];
        }
    }
}

// One thread per quadrature point: points = fold(s(zeta_q)), charges = w_q dt s'(zeta_q) on the
// segment to the right of node i (pointdata_impl.jl:93-103).
// delta^-_k = delta^+ of the previous node (the length of the same segment).
__global__ void dm_from_prev_kernel(int64_t Np, const int32_t* __restrict__ idx_prev, const double* __restrict__ dp,
                                    double* __restrict__ dm) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < Np) dm[k] = dp[idx_prev[k]];
}

__global__ void __launch_bounds__(128) quad_points_kernel(
    KParams K, int64_t Np, const int64_t* __restrict__ offsets, const int32_t* __restrict__ fil_of_node,
    const double* __restrict__ knots, const double* __restrict__ periods, const double* __restrict__ coef,
    const double* __restrict__ dcoef1, double* __restrict__ points, double* __restrict__ charges,
    const double* __restrict__ foff) {
    const int64_t Nq = Np * K.nquad;
    const int64_t mq = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (mq >= Nq) return;
    const int64_t k = mq / K.nquad;
    const int q = (int)(mq - k * K.nquad);
    const int fidx = fil_of_node[k];
    const int64_t off = offsets[fidx];
    const int n = (int)(offsets[fidx + 1] - off);
    const int i = (int)(k - off);
    const FilView f = fil_view(knots, periods, foff, off, n, fidx);
    double s[3], sp[3];
    eval_seg<0>(f, coef + 3 * off, i, K.qz[q], s);
    eval_seg<1>(f, dcoef1 + 3 * off, i, K.qz[q], sp);
    const double dt = knot_at(f, i + 1) - knot_at(f, i);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        points[d * Nq + mq] = fold(s[d], K.L[d], K.open_domain);
        charges[d * Nq + mq] = K.qw[q] * dt * sp[d];
    }
}

}  // namespace

// Shared-memory work space of the spline solve for filaments of at most nmax nodes (4 warps per
// block, 12 doubles per node each); 0 when it does not fit and the global scratch is used.
// Filaments (warps) per spline-solve block: with 2, a 200-node filament's 19 KB of work space per warp
// lets 5 blocks (10 warps) share an SM; with 4, 2 blocks (8 warps) fit (1M nodes: 0.61 vs 0.66 ms for
// the geometry).
constexpr int kSolveWarps = 2;

static int solve_smem_n(int64_t nmax, size_t* bytes) {
    const size_t b = (size_t)kSolveWarps * 12 * nmax * sizeof(double);
    if (nmax > 0 && b <= 200 * 1024) {
        *bytes = b;
        return (int)nmax;
    }
    *bytes = 0;
    return 0;
}

int geometry_from_filaments(vpbs_handle* h, int64_t nfil, const int64_t* d_offsets, const double* d_nodes,
                            int64_t nmax, bool keep_knots) {
    const int64_t Np = h->Np;
    int rc;
    size_t smem_bytes = 0;
    const int smem_n = solve_smem_n(nmax, &smem_bytes);
    // opt in to the exact size every time (a launch at exactly 48 KB also needs it, and the
    // attribute is per function, not per handle)
    if (smem_bytes > 0 &&
        (rc = check_cuda(h, cudaFuncSetAttribute(spline_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem_bytes), "spline kernel shared memory")))
        return rc;
    if ((rc = ensure(h, h->knots, sizeof(double) * (Np + nfil), "knots"))) return rc;
    if ((rc = ensure(h, h->fil_of_node, sizeof(int32_t) * Np, "fil_of_node"))) return rc;
    if ((rc = ensure(h, h->coefs, sizeof(double) * 3 * Np, "coefs"))) return rc;
    if ((rc = ensure(h, h->dcoef1, sizeof(double) * 3 * Np, "dcoef1"))) return rc;
    if ((rc = ensure(h, h->dcoef2, sizeof(double) * 3 * Np, "dcoef2"))) return rc;
    if ((rc = ensure(h, h->spline_scratch, sizeof(double) * 12 * Np + 64, "spline scratch"))) return rc;
    double* knots = (double*)h->knots.p;
    double* periods = knots + Np;
    int32_t* status = (int32_t*)((double*)h->spline_scratch.p + 12 * Np);
    const double* foff = h->have_fil_offsets ? (const double*)h->fil_off.p : nullptr;
    StageScope st(h, ST_GEOMETRY);
    if ((rc = check_cuda(h, cudaMemsetAsync(status, 0, sizeof(int32_t), h->stream), "memset"))) return rc;
    spline_solve_kernel<<<grid_for(nfil, kSolveWarps), 32 * kSolveWarps, smem_bytes, h->stream>>>(
        nfil, d_offsets, d_nodes, knots, periods, (int32_t*)h->fil_of_node.p, (double*)h->coefs.p,
        (double*)h->dcoef1.p, (double*)h->dcoef2.p, (double*)h->spline_scratch.p, status, smem_n, keep_knots ? 1 : 0,
        foff);
    h->launches++;
    const bool want_li = h->K.lia_fraction > 0;
    // without lia_segment_fraction the point-data kernel also writes the quadrature points
    // and charges (one pass of spline evaluations per segment instead of two)
    const bool fuse = !want_li;
    (fuse ? point_data_kernel<true> : point_data_kernel<false>)<<<grid_for(Np, 128), 128, 0, h->stream>>>(
        h->K, Np, d_offsets, (const int32_t*)h->fil_of_node.p, d_nodes, knots, periods, (const double*)h->coefs.p,
        (const double*)h->dcoef1.p, (const double*)h->dcoef2.p, (double*)h->nodes.p, (int32_t*)h->idx_prev.p,
        (double*)h->d1.p, (double*)h->d2.p, (double*)h->dm.p, (double*)h->dp.p, (double*)h->points.p,
        (double*)h->charges.p, (double*)h->li_vel.p, (double*)h->li_psi.p, want_li ? 1 : 0, fuse ? 1 : 0, foff);
    if (fuse)
        dm_from_prev_kernel<<<grid_for(Np, 256), 256, 0, h->stream>>>(Np, (const int32_t*)h->idx_prev.p,
                                                                       (const double*)h->dp.p, (double*)h->dm.p);
    else
        quad_points_kernel<<<grid_for(Np * h->K.nquad, 128), 128, 0, h->stream>>>(
            h->K, Np, d_offsets, (const int32_t*)h->fil_of_node.p, knots, periods, (const double*)h->coefs.p,
            (const double*)h->dcoef1.p, (double*)h->points.p, (double*)h->charges.p, foff);
    h->launches += 2;
    return check_cuda(h, cudaGetLastError(), "geometry kernels");
}

}  // namespace vpbs

// ---------------------------------------------------------------------------------------------
// Allocation-free point data (vpbs_point_data_noalloc).
//
// For callers that cannot allocate device memory themselves or through this library: code
// that runs where cudaMalloc is forbidden or unsafe (inside a stream-ordered region of another
// runtime, under an external memory pool that owns all device memory, or in a host language
// binding that only hands over pre-allocated buffers).  The intermediate arrays of the spline
// solve (knots, B-spline coefficients, the banded factorisation) live in one file-scope device
// array of fixed size instead of cudaMalloc'd buffers; every GPU that loads the library holds
// this array (about 6 MB) until the process exits.
// ---------------------------------------------------------------------------------------------
namespace {

constexpr int64_t kNoAllocMaxNodes = VPBS_NOALLOC_MAX_NODES;
constexpr int64_t kNoAllocMaxFil = VPBS_NOALLOC_MAX_FILAMENTS;
// layout (in doubles): offsets (int64) | knots + periods | fil_of_node (int32) | coefs |
// dcoef1 | dcoef2 | spline scratch (12 per node) | status
constexpr int64_t kNoAllocDoubles =
    (kNoAllocMaxFil + 1) + (kNoAllocMaxNodes + kNoAllocMaxFil) + (kNoAllocMaxNodes + 1) / 2 + 9 * kNoAllocMaxNodes +
    12 * kNoAllocMaxNodes + 8;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Device address of g_noalloc_scratch on the current device.  In host code the symbol itself is
// only a host-side stand-in, never a device address.  The address is looked up on every call (a
// cheap host query once the module is loaded, and it allocates nothing): a cached address would
// go stale if the caller reset the device and the module were loaded again elsewhere.
int noalloc_scratch(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return vpbs::set_error(nullptr, VPBS_ERR_CUDA,
                               std::string("vpbs_point_data_noalloc: cudaGetSymbolAddress failed: ") +
                                   cudaGetErrorString(e));
    *out = (double*)p;
    return 0;
}

// Device memory of `device` (or managed memory) that the kernels may read and write.
bool on_device(const void* p, int device) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // clear the (non-sticky) error so that later calls do not report it
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

// Restores the caller's current device when the entry point returns.
struct DeviceRestore {
    int prev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceRestore() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int vpbs_point_data_noalloc(const vpbs_params* params, int64_t nfil, const int64_t* offsets,
                                       const double* nodes_xyz, void* stream, double* nodes, int32_t* node_idx_prev,
                                       double* deriv1, double* deriv2, double* delta_minus, double* delta_plus,
                                       double* points, double* charges) {
    using namespace vpbs;
    if (!params || !offsets || !nodes_xyz || !nodes || !node_idx_prev || !deriv1 || !deriv2 || !delta_minus ||
        !delta_plus || !points || !charges)
        return set_error(nullptr, VPBS_ERR_ARG, "vpbs_point_data_noalloc: null argument");
    const vpbs_params& P = *params;
    if (nfil < 1 || offsets[0] != 0) return set_error(nullptr, VPBS_ERR_ARG, "vpbs_point_data_noalloc: bad offsets");
    for (int64_t f = 0; f < nfil; ++f)
        if (offsets[f + 1] - offsets[f] < 5)
            return set_error(nullptr, VPBS_ERR_ARG, "each filament needs at least 5 nodes (quintic splines)");
    const int64_t Np = offsets[nfil];
    if (nfil > kNoAllocMaxFil || Np > kNoAllocMaxNodes)
        return set_error(nullptr, VPBS_ERR_ARG,
                         "vpbs_point_data_noalloc: at most " + std::to_string(kNoAllocMaxNodes) + " nodes and " +
                             std::to_string(kNoAllocMaxFil) + " filaments (got " + std::to_string(Np) + " nodes, " +
                             std::to_string(nfil) + " filaments); use vpbs_set_filaments for larger systems");
    if (P.nquad < 1 || P.nquad > kMaxQuad) return set_error(nullptr, VPBS_ERR_PARAMS, "nquad must be in 1:16");
    if (P.lia_segment_fraction > 1.0) return set_error(nullptr, VPBS_ERR_PARAMS, "lia_segment_fraction must be in (0, 1]");
    KParams K{};
    K.Gamma = P.Gamma;
    K.open_domain = (P.splitting == VPBS_SPLITTING_KAISER_BESSEL || P.alpha > 0) ? 0 : 1;
    for (int d = 0; d < 3; ++d) {
        K.L[d] = K.open_domain ? 0.0 : P.L[d];
        K.Lh[d] = K.L[d] / 2;
        if (!K.open_domain && !(P.L[d] > 0)) return set_error(nullptr, VPBS_ERR_PARAMS, "periods L must be positive");
    }
    K.nquad = P.nquad;
    for (int q = 0; q < P.nquad; ++q) { K.qz[q] = P.quad_zeta[q]; K.qw[q] = P.quad_w[q]; }
    K.nquad_near = K.nquad;
    K.lia_fraction = P.lia_segment_fraction > 0 ? P.lia_segment_fraction : 0.0;
    DeviceRestore restore;
    if (cudaSetDevice(P.device) != cudaSuccess)
        return set_error(nullptr, VPBS_ERR_CUDA, "vpbs_point_data_noalloc: cudaSetDevice failed");
    const void* dev_ptrs[] = {nodes_xyz, nodes, node_idx_prev, deriv1, deriv2, delta_minus, delta_plus, points, charges};
    for (const void* p : dev_ptrs)
        if (!on_device(p, P.device))
            return set_error(nullptr, VPBS_ERR_ARG,
                             "vpbs_point_data_noalloc: node and output arrays must be device memory of params->device (" +
                                 std::to_string(P.device) + ")");
    double* base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    int64_t* d_offsets = (int64_t*)base;
    double* knots = base + (kNoAllocMaxFil + 1);
    double* periods = knots + Np;
    int32_t* fil_of_node = (int32_t*)(knots + kNoAllocMaxNodes + kNoAllocMaxFil);
    double* coefs = knots + kNoAllocMaxNodes + kNoAllocMaxFil + (kNoAllocMaxNodes + 1) / 2;
    double* dcoef1 = coefs + 3 * kNoAllocMaxNodes;
    double* dcoef2 = dcoef1 + 3 * kNoAllocMaxNodes;
    double* scratch = dcoef2 + 3 * kNoAllocMaxNodes;
    int32_t* status = (int32_t*)(scratch + 12 * kNoAllocMaxNodes);
    cudaError_t e = cudaMemcpyAsync(d_offsets, offsets, sizeof(int64_t) * (nfil + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int32_t), s);  // the array keeps the last call's data
    if (e != cudaSuccess)
        return set_error(nullptr, VPBS_ERR_CUDA, std::string("vpbs_point_data_noalloc: ") + cudaGetErrorString(e));
    spline_solve_kernel<<<grid_for(nfil, 4), 128, 0, s>>>(nfil, d_offsets, nodes_xyz, knots, periods, fil_of_node, coefs,
                                                          dcoef1, dcoef2, scratch, status, 0, 0, nullptr);
    point_data_kernel<false><<<grid_for(Np, 128), 128, 0, s>>>(K, Np, d_offsets, fil_of_node, nodes_xyz, knots, periods, coefs,
                                                        dcoef1, dcoef2, nodes, node_idx_prev, deriv1, deriv2,
                                                        delta_minus, delta_plus, points, charges, nullptr, nullptr, 0,
                                                        0, nullptr);
    quad_points_kernel<<<grid_for(Np * K.nquad, 128), 128, 0, s>>>(K, Np, d_offsets, fil_of_node, knots, periods, coefs,
                                                                   dcoef1, points, charges, nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(nullptr, VPBS_ERR_CUDA, std::string("vpbs_point_data_noalloc: ") + cudaGetErrorString(e));
    return 0;
}
