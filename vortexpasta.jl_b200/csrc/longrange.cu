// Long-range part of the Ewald split on the device (src/BiotSavart/longrange/longrange.jl,
// longrange/backends/nonuniformffts.jl):
//  1. type-1 NUFFT of the quadrature charges: exponential-of-semicircle (ES) kernel spreading
//     onto the oversampled grid (Barnett, Magland & af Klinteberg, SIAM J. Sci. Comput. 2019),
//     then a batched 3-D real-to-complex FFT (cuFFT);
//  2. one fused Fourier-space kernel: deconvolution, Gamma/V prefactor, Hermitian-symmetry
//     zeroing (longrange.jl:556-583), optional spherical truncation (longrange.jl:497-532),
//     the vorticity coefficients kept for get_longrange_field_fourier, and the
//     streamfunction (longrange.jl:102-125) / Biot-Savart (longrange.jl:128-142) operators
//     times the Ewald Gaussian exp(-k^2/4 alpha^2) (cache_common.jl:64-76) and the type-2
//     deconvolution, written straight into the complex-to-real FFT input;
//  3. batched complex-to-real FFT and ES-kernel interpolation at the nodes (type 2).
#include <cmath>
#include <type_traits>
#include <vector>

#include "vpbs_internal.cuh"
#include "tc_sm100.cuh"

namespace vpbs {

// Gauss-Legendre rule on [-1, 1] by Newton iteration on P_n (host).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.resize(n);
    w.resize(n);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

namespace {


// Fourier transform of the spreading kernel at frequency xi (radians per grid spacing), both kernels
// shifted down by their edge value so that they vanish at |u| = m (r = sqrt(1 - (u/m)^2)):
//   ES (exponential of semicircle): psi(u) = exp(beta (r - 1)) - e^{-beta};
//   backward Kaiser-Bessel:         psi(u) = sinh(beta r) / (r sinh beta) - beta / sinh beta.
// With u = m sin t (r = cos t) the transform is m int_{-pi/2}^{pi/2} psi(m sin t) cos(xi m sin t) cos t dt,
// a smooth integrand, evaluated with a 128-point Gauss-Legendre rule.
double es_hat(double xi, int m, double beta, int kind) {
    static std::vector<double> gx, gw;
    if (gx.empty()) gauss_legendre(128, gx, gw);
    double s = 0.0;
    for (size_t i = 0; i < gx.size(); ++i) {
        const double th = 0.5 * kPi * gx[i], c = std::cos(th);
        const double pc = kind == VPBS_NUFFT_KAISER_BESSEL
                              ? std::sinh(beta * c) / std::sinh(beta) - (beta / std::sinh(beta)) * c
                              : (std::exp(beta * (c - 1.0)) - std::exp(-beta)) * c;
        s += 0.5 * kPi * gw[i] * pc * std::cos(xi * m * std::sin(th));
    }
    return m * s;
}

inline int mode_of(int i, int N) { return i < (N + 1) / 2 ? i : i - N; }

// ES kernel shifted down by its edge value e^{-beta} (passed as `edge`) so that it vanishes
// continuously at |u| = m: which 2m-point window a point on a grid node gets then no longer
// depends on the last bit of its coordinate.
__device__ __forceinline__ double es_kernel(double u, int m, double beta, double edge, int kind) {
    double z = u / m;
    double s = 1.0 - z * z;
    if (!(s > 0.0)) return 0.0;
    if (kind == VPBS_NUFFT_KAISER_BESSEL) {
        // backward Kaiser-Bessel kernel sinh(beta r) / (r sinh beta), less its edge value beta / sinh beta
        const double r = sqrt(s);
        return (r > 1e-12 ? sinh(beta * r) / (r * sinh(beta)) : beta / sinh(beta)) - edge;
    }
    return exp(beta * (sqrt(s) - 1.0)) - edge;
}

__device__ __forceinline__ int wrapi(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// i mod n for i in [-n, 2n) without a division (a folded footprint start plus s < 2m <= n).
__device__ __forceinline__ int wrap1(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// es_kernel for a compile-time width W = 2m: u / m as a product with the constant 2 / W.
template <int W>
__device__ __forceinline__ double es_kernel_w(double u, double beta, double edge, int kind) {
    constexpr double inv_m = 2.0 / W;
    const double z = u * inv_m;
    const double s = 1.0 - z * z;
    if (!(s > 0.0)) return 0.0;
    if (kind == VPBS_NUFFT_KAISER_BESSEL) {
        const double r = sqrt(s);
        return (r > 1e-12 ? sinh(beta * r) / (r * sinh(beta)) : beta / sinh(beta)) - edge;
    }
    return exp(beta * (sqrt(s) - 1.0)) - edge;
}

constexpr int kSpreadBatch = 32;

// Complex value of the grid precision T from double parts.
template <typename C>
__device__ __forceinline__ C mkc(double x, double y);
template <>
__device__ __forceinline__ double2 mkc<double2>(double x, double y) { return make_double2(x, y); }
template <>
__device__ __forceinline__ float2 mkc<float2>(double x, double y) { return make_float2((float)x, (float)y); }

// Type-1 spreading with global atomics (fallback when the grid cannot be tiled into bricks):
// each block takes kSpreadBatch points; kernel values are tabulated in shared memory, then
// every thread adds the charges along x-lines of the (2m)^3 footprint.
template <typename T>
__global__ void __launch_bounds__(256) spread_kernel_atomic(
    LRSizes S, int64_t Nq, const double* __restrict__ src, double sx0, double sx1, double sx2,
    T* __restrict__ grid) {
    __shared__ double phi[kSpreadBatch][3][2 * kMaxHalfSupport];
    __shared__ int i0s[kSpreadBatch][3];
    __shared__ double qs[kSpreadBatch][3];
    const int w = 2 * S.m;
    const int64_t pbase = (int64_t)blockIdx.x * kSpreadBatch;
    const int np = (int)((Nq - pbase) < kSpreadBatch ? (Nq - pbase) : kSpreadBatch);
    const double scale[3] = {sx0, sx1, sx2};
    for (int idx = threadIdx.x; idx < np * 3; idx += blockDim.x) {
        const int p = idx / 3, d = idx % 3;
        const int64_t j = pbase + p;
        const double h = 2.0 * kPi / S.n[d];
        const double xh = (src[d * Nq + j] * scale[d]) / h;
        const int i0 = (int)floor(xh) - S.m + 1;
        i0s[p][d] = i0;
        for (int s = 0; s < w; ++s) phi[p][d][s] = es_kernel(xh - (i0 + s), S.m, S.beta, S.edge, S.kernel);
        qs[p][d] = src[(3 + d) * Nq + j];
    }
    __syncthreads();
    const int per = w * w;
    const int64_t ng = S.ngrid;
    for (int item = threadIdx.x; item < np * per; item += blockDim.x) {
        const int p = item / per, l = item % per;
        const int sy = l % w, sz = l / w;
        const int iz = wrapi(i0s[p][2] + sz, S.n[2]);
        const int iy = wrapi(i0s[p][1] + sy, S.n[1]);
        const double fyz = phi[p][2][sz] * phi[p][1][sy];
        const double q0 = qs[p][0] * fyz, q1 = qs[p][1] * fyz, q2 = qs[p][2] * fyz;
        const int64_t row = ((int64_t)iz * S.n[1] + iy) * S.n[0];
        for (int sx = 0; sx < w; ++sx) {
            const int ix = wrapi(i0s[p][0] + sx, S.n[0]);
            const double f = phi[p][0][sx];
            atomicAdd(grid + row + ix, (T)(q0 * f));
            atomicAdd(grid + ng + row + ix, (T)(q1 * f));
            atomicAdd(grid + 2 * ng + row + ix, (T)(q2 * f));
        }
    }
}

// Fused Fourier-space kernel over the r2c grid [n2][n1][n0/2+1] (C: double2 or float2; the
// arithmetic is FP64 in both forms, only the grids are stored in the grid precision).
template <typename C>
__global__ void __launch_bounds__(256) fourier_kernel(
    LRSizes S, double pref, double k0x, double k0y, double k0z, int truncate, double kmax2, int fields,
    double kb_beta2, double kb_rc2, double kb_c,
    const double* __restrict__ dec0, const double* __restrict__ dec1, const double* __restrict__ dec2,
    const double* __restrict__ decE0, const double* __restrict__ decE1, const double* __restrict__ decE2,
    C* __restrict__ gc, C* __restrict__ gc2, double2* __restrict__ uhat, int store_uhat) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= S.ncgrid) return;
    const int ix = (int)(idx % S.nxc);
    const int64_t rest = idx / S.nxc;
    const int iy = (int)(rest % S.n[1]);
    const int iz = (int)(rest / S.n[1]);
    const int ky = iy < (S.n[1] + 1) / 2 ? iy : iy - S.n[1];
    const int kz = iz < (S.n[2] + 1) / 2 ? iz : iz - S.n[2];
    const int lo1 = -(S.Ns[1] / 2), hi1 = (S.Ns[1] - 1) / 2;
    const int lo2 = -(S.Ns[2] / 2), hi2 = (S.Ns[2] - 1) / 2;
    const bool in_red = ix < S.nkx && ky >= lo1 && ky <= hi1 && kz >= lo2 && kz <= hi2;
    const int64_t cstride = S.ncgrid;
    double2 w[3] = {{0, 0}, {0, 0}, {0, 0}};
    bool live = false;
    if (in_red) {
        const bool zero = (ix == S.nkx - 1) || (S.Ns[1] % 2 == 0 && ky == lo1) || (S.Ns[2] % 2 == 0 && kz == lo2);
        const int ry = ky < 0 ? ky + S.Ns[1] : ky;
        const int rz = kz < 0 ? kz + S.Ns[2] : kz;
        const double kx = k0x * ix, kyy = k0y * ky, kzz = k0z * kz;
        const double k2 = kx * kx + kyy * kyy + kzz * kzz;
        live = !zero && !(truncate && k2 > kmax2);
        if (live) {
            const double f = pref * (dec0[ix] * dec1[ry] * dec2[rz]);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const C F = gc[c * cstride + idx];
                w[c] = make_double2((double)F.x * f, (double)F.y * f);
            }
        }
        if (store_uhat) {
            const int64_t u = ((int64_t)rz * S.Ns[1] + ry) * S.nkx + ix;
#pragma unroll
            for (int c = 0; c < 3; ++c) uhat[c * S.nmodes + u] = w[c];
        }
        if (live) {
            const double k2inv = (k2 == 0.0) ? 0.0 : 1.0 / k2;
            double g = decE0[ix] * decE1[ry] * decE2[rz];
            if (kb_beta2 > 0.0) {
                // Kaiser-Bessel filter (kaiser_bessel.jl:266-278): beta / sinh(beta) sinh(q) / q,
                // q = sqrt(beta^2 - k^2 rcut^2), zero beyond k = beta / rcut
                const double sq = kb_beta2 - k2 * kb_rc2;
                if (sq > 0.0) {
                    const double q = sqrt(sq);
                    g *= kb_c * sinh(q) / q;
                } else {
                    g = 0.0;
                }
            }
            if (fields & VPBS_VELOCITY) {
                // i k x w / k^2 ; (i w).x = -w.y, (i w).y = w.x
                const double2 iw0 = make_double2(-w[0].y, w[0].x), iw1 = make_double2(-w[1].y, w[1].x),
                              iw2 = make_double2(-w[2].y, w[2].x);
                const double fk = k2inv * g;
                gc[idx] = mkc<C>((kyy * iw2.x - kzz * iw1.x) * fk, (kyy * iw2.y - kzz * iw1.y) * fk);
                gc[cstride + idx] = mkc<C>((kzz * iw0.x - kx * iw2.x) * fk, (kzz * iw0.y - kx * iw2.y) * fk);
                gc[2 * cstride + idx] = mkc<C>((kx * iw1.x - kyy * iw0.x) * fk, (kx * iw1.y - kyy * iw0.y) * fk);
            }
            if (fields & VPBS_STREAMFUNCTION) {
                const double fk = k2inv * g;
#pragma unroll
                for (int c = 0; c < 3; ++c) gc2[c * cstride + idx] = mkc<C>(w[c].x * fk, w[c].y * fk);
            }
        }
    }
    if (!live) {
        if (fields & VPBS_VELOCITY)
#pragma unroll
            for (int c = 0; c < 3; ++c) gc[c * cstride + idx] = mkc<C>(0.0, 0.0);
        if (fields & VPBS_STREAMFUNCTION)
#pragma unroll
            for (int c = 0; c < 3; ++c) gc2[c * cstride + idx] = mkc<C>(0.0, 0.0);
    }
}

// ---- brick spreading (no global atomics) ----
// The oversampled grid is tiled into bricks of B^3 points.  Points are binned by the brick
// holding the first grid point of their footprint; a footprint of w <= B points can then only
// reach the brick of its bin and the next one in each direction, so brick b collects the points
// of bins b and b-1 (per dimension, periodic).  Every grid value is written exactly once, with
// plain stores, by the CTA that owns its brick.

__device__ __forceinline__ int footprint_start(double x, double scale, int n, int m) {
    const double xh = (x * scale) / (2.0 * kPi / n);
    return wrapi((int)floor(xh) - m + 1, n);
}

__global__ void spread_bin_count_kernel(LRSizes S, int B, int nb0, int nb1, int nb2, int64_t Nq,
                                        const double* __restrict__ src, double sx0, double sx1, double sx2,
                                        int32_t* __restrict__ bin, int32_t* __restrict__ rank,
                                        int32_t* __restrict__ counts) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Nq) return;
    const int b0 = footprint_start(src[j], sx0, S.n[0], S.m) / B;
    const int b1 = footprint_start(src[Nq + j], sx1, S.n[1], S.m) / B;
    const int b2 = footprint_start(src[2 * Nq + j], sx2, S.n[2], S.m) / B;
    const int32_t b = (b2 * nb1 + b1) * nb0 + b0;
    bin[j] = b;
    rank[j] = warp_aggregated_rank(counts, b);
}

// Scatter the points into bin order, with everything the brick kernel needs per point: the
// wrapped footprint start per dimension, the 3 x w kernel values and the 3 charges.
// binned layout per slot: [3 charges][3 w kernel values] (grid precision T), foot: [3] int32.
// Positions and kernel values are computed in FP64 and stored in T.
template <typename T>
__global__ void spread_bin_scatter_kernel(LRSizes S, int64_t Nq, const double* __restrict__ src, double sx0,
                                          double sx1, double sx2, const int32_t* __restrict__ bin,
                                          const int32_t* __restrict__ rank, const int32_t* __restrict__ start,
                                          T* __restrict__ binned, int32_t* __restrict__ foot) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Nq) return;
    const int64_t pos = (int64_t)start[bin[j]] + rank[j];
    const int w = 2 * S.m;
    const int stride = 3 + 3 * w;
    T* out = binned + pos * stride;
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = (T)src[(3 + c) * Nq + j];
    const double scale[3] = {sx0, sx1, sx2};
    for (int d = 0; d < 3; ++d) {
        const double xh = (src[d * Nq + j] * scale[d]) / (2.0 * kPi / S.n[d]);
        const int i0 = (int)floor(xh) - S.m + 1;
        foot[3 * pos + d] = wrapi(i0, S.n[d]);
        for (int s = 0; s < w; ++s) out[3 + d * w + s] = (T)es_kernel(xh - (i0 + s), S.m, S.beta, S.edge, S.kernel);
    }
}

// Shared-memory brick spreading: one CTA per brick keeps the brick's three components in
// shared memory (x rows padded to B+1 against bank conflicts), adds the part of every nearby
// footprint that falls inside the brick with shared-memory atomics (one warp per point, lanes
// over the footprint's (y, z) lines), then writes the brick to the grid with plain stores.
constexpr int kBrickThreads = 256;

template <int B, typename T>
__global__ void __launch_bounds__(kBrickThreads) spread_brick_kernel(
    LRSizes S, int nb0, int nb1, int nb2, const int32_t* __restrict__ bin_start, const T* __restrict__ binned,
    const int32_t* __restrict__ foot, T* __restrict__ grid) {
    extern __shared__ __align__(16) unsigned char tile_raw[];
    T* tile = reinterpret_cast<T*>(tile_raw);  // [3][B][PZ] with rows of RX values
    __shared__ T phw[kBrickThreads / 32][3 + 6 * kMaxHalfSupport];
    constexpr int RX = B + 1;        // x-row stride (bank spread along y)
    constexpr int PZ = B * RX + 8;   // z-plane stride (16-word bank shift between planes)
    constexpr int TC = B * PZ;       // doubles per component
    const int w = 2 * S.m;
    const int stride = 3 + 3 * w;
    const int bx = blockIdx.x % nb0;
    const int by = (blockIdx.x / nb0) % nb1;
    const int bz = blockIdx.x / (nb0 * nb1);
    const int bs[3] = {bx * B, by * B, bz * B};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 3 * TC; i += kBrickThreads) tile[i] = (T)0;
    __syncthreads();
    T* ph = phw[warp];  // [q0 q1 q2 | phi_x[w] | phi_y[w] | phi_z[w]]
    for (int nbr = 0; nbr < 8; ++nbr) {
        const int cx = (bx - (nbr & 1) + nb0) % nb0;
        const int cy = (by - ((nbr >> 1) & 1) + nb1) % nb1;
        const int cz = (bz - ((nbr >> 2) & 1) + nb2) % nb2;
        const int b = (cz * nb1 + cy) * nb0 + cx;
        const int64_t p1 = bin_start[b + 1];
        for (int64_t j = bin_start[b] + warp; j < p1; j += kBrickThreads / 32) {
            // footprint offset relative to the brick (periodic) and overlap range, per dimension
            int o[3], lo[3], hi[3];
            bool empty = false;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                o[d] = foot[3 * j + d] - bs[d];
                if (o[d] >= B) o[d] -= S.n[d];
                lo[d] = o[d] < 0 ? -o[d] : 0;
                hi[d] = B - o[d] < w ? B - o[d] : w;
                empty = empty || lo[d] >= hi[d];
            }
            if (empty) continue;  // warp-uniform
            for (int it = lane; it < stride; it += 32) ph[it] = binned[j * stride + it];
            __syncwarp();
            const T q0 = ph[0], q1 = ph[1], q2 = ph[2];
            const T* phx = ph + 3;
            const T* phy = phx + w;
            const T* phz = phy + w;
            const int ny = hi[1] - lo[1], nz = hi[2] - lo[2];
            for (int l = lane; l < ny * nz; l += 32) {
                const int sy = lo[1] + l % ny, sz = lo[2] + l / ny;
                const T f = phy[sy] * phz[sz];
                T* row = tile + (o[2] + sz) * PZ + (o[1] + sy) * RX + o[0];
                for (int sx = lo[0]; sx < hi[0]; ++sx) {
                    const T g = f * phx[sx];
                    atomicAdd(row + sx, q0 * g);
                    atomicAdd(row + TC + sx, q1 * g);
                    atomicAdd(row + 2 * TC + sx, q2 * g);
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    const int64_t ng = S.ngrid;
    for (int i = threadIdx.x; i < 3 * B * B * B; i += kBrickThreads) {
        const int c = i / (B * B * B), r = i % (B * B * B);
        const int x = r % B, y = (r / B) % B, z = r / (B * B);
        grid[c * ng + ((int64_t)(bs[2] + z) * S.n[1] + (bs[1] + y)) * S.n[0] + bs[0] + x] =
            tile[c * TC + z * PZ + y * RX + x];
    }
}

// Plane-owner brick spreading for FP32 grids and narrow kernels (w = 2m <= 8), 16^3 bricks, no
// atomics: one CTA of 16 warps per brick, warp z owning the brick's z-plane z in shared memory.
// The candidate points (those of the 8 bins whose footprints can reach the brick) are tested one
// per thread and only the overlapping ones are staged, in batches, as brick-aligned, zero-padded
// kernel rows (px, py, pz of 16 values; 8 threads per point) together with one slot list per
// plane.  Each warp then walks the list of its plane and adds, for every listed point, a P x P
// patch of (x, y) cells starting at the footprint corner (P = 4 for w <= 4, 8 for w <= 8; cells
// past the footprint multiply a zero kernel value) with plain read-modify-writes: the plane has
// one writer and the lanes of one instruction hold distinct cells.  The x-row stride RX puts the 32 / P rows of one instruction
// in disjoint banks (RX = 24 for P = 8: row offsets 0, 24, 16, 8; RX = 20 for P = 4).
// Measured on the B200: FP32 shared atomicAdd sustains 2.0 T updates/s conflict-free against
// 4.2 T for plain read-modify-writes, and the per-point work (footprint tests, kernel rows) is
// done once per point and batch instead of by every lane of a warp.  Variants measured slower
// on the 1M-node tangle (m = 4, spread 5.9 ms here): float4 cells (one 16-byte load and store
// per update, 8 instead of 6 shared wavefronts: 6.2 ms), the plane held in registers (lane per
// column, 8 rows of 3 components: more instructions per point, 8.3 ms) and a warp-uniform skip
// of patch iterations whose rows miss the brick (6.3 ms).
constexpr int kPlaneB = 16;
constexpr int kPlaneThreads = 512;
constexpr int kPlaneBatch = 128;

template <int P>
struct PlaneLayout {
    static constexpr int RX = P == 8 ? 24 : 20;  // x-row stride
    static constexpr int PL = kPlaneB * RX;      // z-plane stride
    static constexpr int TC = kPlaneB * PL;      // floats per component
};

// One staged point: charges, the w kernel values per dimension zero-padded to P entries, and the
// footprint corner in brick coordinates (may be negative).
template <int P>
struct __align__(16) PlaneSlot {
    float q[4];
    float px[P], py[P], pz[P];
    int xs, ys, zs, pad;
};

template <int P>
__global__ void __launch_bounds__(kPlaneThreads, 2) spread_plane_kernel(
    LRSizes S, int nb0, int nb1, int nb2, const int32_t* __restrict__ bin_start, const float* __restrict__ binned,
    const int32_t* __restrict__ foot, float* __restrict__ grid) {
    using Lay = PlaneLayout<P>;
    extern __shared__ __align__(16) float ptile[];  // [3][16 planes][16 rows][RX]
    __shared__ PlaneSlot<P> slot[kPlaneBatch];
    __shared__ int32_t pend_j[kPlaneThreads];        // overlapping candidates of the current chunk
    __shared__ int16_t pend_o[kPlaneThreads][3];     // their footprint corners (brick coordinates)
    __shared__ uint8_t plist[kPlaneB][kPlaneBatch];  // slots covering each plane
    __shared__ int pcount[kPlaneB];
    __shared__ int npend;
    __shared__ int nbin_start[8], nbin_base[9];
    const int w = 2 * S.m;
    const int stride = 3 + 3 * w;
    const int bx = blockIdx.x % nb0;
    const int by = (blockIdx.x / nb0) % nb1;
    const int bz = blockIdx.x / (nb0 * nb1);
    const int bs[3] = {bx * kPlaneB, by * kPlaneB, bz * kPlaneB};
    const int lane = threadIdx.x & 31, z = threadIdx.x >> 5;  // warp z owns plane z
    for (int i = threadIdx.x; i < 3 * Lay::TC; i += kPlaneThreads) ptile[i] = 0.0f;
    if (threadIdx.x < 8) {
        const int nbr = threadIdx.x;
        const int cx = (bx - (nbr & 1) + nb0) % nb0;
        const int cy = (by - ((nbr >> 1) & 1) + nb1) % nb1;
        const int cz = (bz - ((nbr >> 2) & 1) + nb2) % nb2;
        const int b = (cz * nb1 + cy) * nb0 + cx;
        nbin_start[nbr] = bin_start[b];
        nbin_base[nbr + 1] = bin_start[b + 1] - bin_start[b];
    }
    if (threadIdx.x < kPlaneB) pcount[threadIdx.x] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        nbin_base[0] = 0;
        for (int k = 1; k <= 8; ++k) nbin_base[k] += nbin_base[k - 1];
    }
    __syncthreads();
    const int ntot = nbin_base[8];
    // this lane's cells of the P x P patch: (cell % P, cell / P) for cell = lane + 32 it
    constexpr int kIter = (P * P + 31) / 32;
    int cxo[kIter], cyo[kIter];
#pragma unroll
    for (int it = 0; it < kIter; ++it) {
        const int cell = lane + 32 * it;
        cxo[it] = cell % P;
        cyo[it] = cell < P * P ? cell / P : 0;
    }
    const bool live0 = lane < P * P;  // lanes past the patch (P = 4: 16 cells) stay idle
    float* plane = ptile + z * Lay::PL;
    for (int c0 = 0; c0 < ntot; c0 += kPlaneThreads) {
        // ---- 1: keep the candidates of this chunk whose footprint meets the brick ----
        if (threadIdx.x == 0) npend = 0;
        __syncthreads();
        {
            const int k = c0 + threadIdx.x;
            if (k < ntot) {
                int nb = 0;
#pragma unroll
                for (int i = 1; i < 8; ++i) nb += k >= nbin_base[i];
                const int32_t j = nbin_start[nb] + (k - nbin_base[nb]);
                int o[3];
                bool empty = false;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    o[d] = foot[3 * (int64_t)j + d] - bs[d];
                    if (o[d] >= kPlaneB) o[d] -= S.n[d];
                    empty = empty || o[d] + w <= 0 || o[d] >= kPlaneB;
                }
                if (!empty) {
                    const int q = atomicAdd(&npend, 1);
                    pend_j[q] = j;
#pragma unroll
                    for (int d = 0; d < 3; ++d) pend_o[q][d] = (int16_t)o[d];
                }
            }
        }
        __syncthreads();
        const int np = npend;
        for (int p0 = 0; p0 < np; p0 += kPlaneBatch) {
            const int nbatch = np - p0 < kPlaneBatch ? np - p0 : kPlaneBatch;
            // ---- 2: stage the points (4 threads per slot) and the per-plane slot lists ----
            {
                const int sidx = threadIdx.x >> 2, part = threadIdx.x & 3;
                if (sidx < nbatch) {
                    PlaneSlot<P>& sl = slot[sidx];
                    const int q = p0 + sidx;
                    const float* src = binned + (int64_t)pend_j[q] * stride;
                    // part d < 3: kernel row d (w values, zero-padded to P); part 3: charges, corner
                    if (part < 3) {
                        float* row = part == 0 ? sl.px : part == 1 ? sl.py : sl.pz;
#pragma unroll
                        for (int r = 0; r < P; ++r) row[r] = r < w ? src[3 + part * w + r] : 0.0f;
                    } else {
                        sl.q[0] = src[0];
                        sl.q[1] = src[1];
                        sl.q[2] = src[2];
                        sl.xs = pend_o[q][0];
                        sl.ys = pend_o[q][1];
                        sl.zs = pend_o[q][2];
                    }
                    // planes [max(o2, 0), min(o2 + w, 16)), split over the slot's 4 threads
                    const int o2 = pend_o[q][2];
                    const int zlo = o2 < 0 ? 0 : o2, zhi = o2 + w < kPlaneB ? o2 + w : kPlaneB;
                    for (int zz = zlo + part; zz < zhi; zz += 4) {
                        const int pos = atomicAdd(&pcount[zz], 1);
                        plist[zz][pos] = (uint8_t)sidx;
                    }
                }
            }
            __syncthreads();
            // ---- 3: warp z adds the patches of the slots covering plane z ----
            const int nz = pcount[z];
            for (int t = 0; t < nz; ++t) {
                const PlaneSlot<P>& sl = slot[plist[z][t]];
                const float fz = sl.pz[z - sl.zs];
                const float a0 = sl.q[0] * fz, a1 = sl.q[1] * fz, a2 = sl.q[2] * fz;
                const int xs = sl.xs, ys = sl.ys;
#pragma unroll
                for (int it = 0; it < kIter; ++it) {
                    const int cx = xs + cxo[it], cy = ys + cyo[it];
                    if (live0 && (unsigned)cx < (unsigned)kPlaneB && (unsigned)cy < (unsigned)kPlaneB) {
                        const float g = sl.px[cxo[it]] * sl.py[cyo[it]];
                        float* cell = plane + cy * Lay::RX + cx;
                        cell[0] = fmaf(a0, g, cell[0]);
                        cell[Lay::TC] = fmaf(a1, g, cell[Lay::TC]);
                        cell[2 * Lay::TC] = fmaf(a2, g, cell[2 * Lay::TC]);
                    }
                }
            }
            if (lane == 0) pcount[z] = 0;  // read above by this warp only; refilled after the barrier
            __syncthreads();
        }
    }
    const int64_t ng = S.ngrid;
    for (int i = threadIdx.x; i < 3 * kPlaneB * kPlaneB * kPlaneB; i += kPlaneThreads) {
        const int c = i / (kPlaneB * kPlaneB * kPlaneB), r = i % (kPlaneB * kPlaneB * kPlaneB);
        const int x = r % kPlaneB, y = (r / kPlaneB) % kPlaneB, zz = r / (kPlaneB * kPlaneB);
        grid[c * ng + ((int64_t)(bs[2] + zz) * S.n[1] + (bs[1] + y)) * S.n[0] + bs[0] + x] =
            ptile[c * Lay::TC + zz * Lay::PL + y * Lay::RX + x];
    }
}

// ---- Tensor-core spreading (FP32 grids, NUFFT half-support m <= 4, bricks of 16^3) ----
// The spread onto one brick is a dense product over the points p whose footprint meets it:
//   grid[c][z][y][x] = sum_p (q_pc phi_z,p(z)) (phi_y,p(y) phi_x,p(x)),
// i.e. D[(y, x), (c, z)] = sum_p A[(y, x), p] B[(c, z), p] with M = 256 rows in two halves of 128
// (y < 8, y >= 8), N = 48 columns and K = the points, 16 per batch.  A pre-pass writes one record
// per (point, brick) pair, grouped by brick: charges, the footprint corner relative to the brick and
// the kernel values (computed once per point).  The brick's kernel streams its records into shared
// memory with bulk copies (double-buffered), builds the operands there (K-major core matrices of 8
// rows x 4 values; A holds only the current footprints, cleared again before reuse) and multiplies
// them with tcgen05.mma kind::tf32 into two FP32 accumulators in tensor memory.  Each operand is split
// into TF32 hi + lo parts and D accumulates hi*hi + hi*lo + lo*hi (3xTF32: FP32 accuracy, ~1e-7
// relative).  Operand buffers are double-buffered: the tensor cores multiply batch b while the threads
// build batch b + 1; mbarriers signalled by tcgen05.commit guard their reuse.  The brick's cells are
// then read from tensor memory and written once (no atomics).  Every wait is bounded: on a timeout the
// kernel records it in *status, stops issuing, and releases its tensor memory.
constexpr int kTcThreads = 384;  // warp 0 issues; 11 builder warps
constexpr int kTcKB = 16;      // points per batch: two K-steps of 8
constexpr int kTcChunk = 128;  // records per bulk copy (a multiple of kTcKB: batches never straddle chunks)
constexpr int kTcBatchesPerChunk = kTcChunk / kTcKB;
constexpr int kTcRecMax = 28;  // floats per record for w <= 8
constexpr int kTcBuilderWarps = kTcThreads / 32 - 1;  // warps 1..W/2 write A, the others B
constexpr uint32_t kTcWaitLimit = 1u << 26;

// floats per record: charges (3), packed corner (1), 3 kernel rows of w values, padded to 16 bytes
__host__ __device__ constexpr int tc_record_floats(int w) { return (4 + 3 * w + 3) & ~3; }

__device__ __forceinline__ void tc_point_bricks(const int f[3], int w, int b0[3], int two[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        b0[d] = f[d] >> 4;
        two[d] = (f[d] & 15) + w > 16;
    }
}

// Records per brick (counting pass): every brick a point's footprint meets.
__global__ void tc_rec_count_kernel(LRSizes S, int nb0, int nb1, int nb2, int64_t Nq, const double* __restrict__ src,
                                    double sx0, double sx1, double sx2, int32_t* __restrict__ counts) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Nq) return;
    const int w = 2 * S.m;
    const int f[3] = {footprint_start(src[j], sx0, S.n[0], S.m), footprint_start(src[Nq + j], sx1, S.n[1], S.m),
                      footprint_start(src[2 * Nq + j], sx2, S.n[2], S.m)};
    int b0[3], two[3];
    tc_point_bricks(f, w, b0, two);
    const int nbv[3] = {nb0, nb1, nb2};
    for (int e = 0; e < 8; ++e) {
        const int ex = e & 1, ey = (e >> 1) & 1, ez = e >> 2;
        if ((ex && !two[0]) || (ey && !two[1]) || (ez && !two[2])) continue;
        const int bx = (b0[0] + ex) % nbv[0], by = (b0[1] + ey) % nbv[1], bz = (b0[2] + ez) % nbv[2];
        warp_aggregated_rank(counts, (bz * nb1 + by) * nb0 + bx);
    }
}

// The records: position start[brick] + rank (ranks from a second aggregated count into `fill`).  A
// record is assembled in registers and written with 16-byte stores.
template <int W>
__global__ void __launch_bounds__(128) tc_rec_scatter_kernel(LRSizes S, int nb0, int nb1, int nb2, int64_t Nq,
                                                             const double* __restrict__ src, double sx0, double sx1,
                                                             double sx2, const int32_t* __restrict__ start,
                                                             int32_t* __restrict__ fill, float* __restrict__ rec) {
    constexpr int R = tc_record_floats(W);
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Nq) return;
    const double scale[3] = {sx0, sx1, sx2};
    int f[3];
    float r[R];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double xh = (src[d * Nq + j] * scale[d]) / (2.0 * kPi / S.n[d]);
        const int i0 = (int)floor(xh) - S.m + 1;
        f[d] = wrapi(i0, S.n[d]);
#pragma unroll
        for (int s = 0; s < W; ++s) r[4 + d * W + s] = (float)es_kernel_w<W>(xh - (i0 + s), S.beta, S.edge, S.kernel);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c] = (float)src[(3 + c) * Nq + j];
#pragma unroll
    for (int k = 4 + 3 * W; k < R; ++k) r[k] = 0.0f;
    int b0[3], two[3];
    tc_point_bricks(f, W, b0, two);
    const int nbv[3] = {nb0, nb1, nb2};
    for (int e = 0; e < 8; ++e) {
        const int ex = e & 1, ey = (e >> 1) & 1, ez = e >> 2;
        if ((ex && !two[0]) || (ey && !two[1]) || (ez && !two[2])) continue;
        const int bx = (b0[0] + ex) % nbv[0], by = (b0[1] + ey) % nbv[1], bz = (b0[2] + ez) % nbv[2];
        const int32_t b = (bz * nb1 + by) * nb0 + bx;
        const int64_t pos = (int64_t)start[b] + warp_aggregated_rank(fill, b);
        // corner relative to the brick, biased by 64 into one byte per dimension
        const int ox = (f[0] & 15) - 16 * ex, oy = (f[1] & 15) - 16 * ey, oz = (f[2] & 15) - 16 * ez;
        r[3] = __int_as_float((ox + 64) | ((oy + 64) << 8) | ((oz + 64) << 16));
        float4* dst = reinterpret_cast<float4*>(rec + pos * R);
#pragma unroll
        for (int k = 0; k < R / 4; ++k) dst[k] = make_float4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
    }
}

struct TcSpreadSmem {
    // operands [stage][hi, lo], K-major core matrices of 8 rows x 4 values.  A: rows m = 16 y + x, the
    // halves y < 8 and y >= 8 one after the other, so the element (y, x, k) sits at
    // 256 y + 128 (x / 8) + 4 (x % 8) + 32 (k / 4) + k % 4; zero outside the footprints of the batch
    // the stage holds (entries are cleared again before the stage is reused).  B: rows n = 16 c + z.
    float A[2][2][256 * kTcKB];
    float B[2][2][48 * kTcKB];
    float pts[2][kTcChunk * kTcRecMax];  // records of the current and the next chunk
    int fail;
    uint64_t full[2];    // operands of each stage written (one arrival per builder warp)
    uint64_t empty[2];   // multiplications of each stage done (tcgen05.commit)
    uint64_t cpbar[2];   // bulk copy of each record buffer done
    uint32_t tslot;
};

// Warp roles: warp 0 (one elected thread) issues the bulk copies of the records and the multiplications;
// warps 1..W/2 write A (W threads per point slot: one x entry each, all y entries), the other builder
// warps write B.
// No CTA-wide barrier inside the loop: builders arrive on full[stage] when their part of a batch is
// written, the issuing thread waits on it, multiplies and commits to empty[stage], which the builders
// wait on before they overwrite that stage two batches later.  A record buffer is refilled (chunk c + 2)
// once the issuing thread has seen every batch of chunk c written, i.e. read by all builders.
template <int W>
__global__ void __launch_bounds__(kTcThreads, 2) spread_tc_kernel(LRSizes S, int nb0, int nb1,
                                                                  const int32_t* __restrict__ rec_start,
                                                                  const float* __restrict__ rec, float* __restrict__ grid,
                                                                  int* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char tc_raw[];
    TcSpreadSmem& T = *reinterpret_cast<TcSpreadSmem*>(tc_raw);
    volatile int* fail = &T.fail;
    constexpr int B16 = 16;
    constexpr int R = tc_record_floats(W);
    const int bx = blockIdx.x % nb0;
    const int by = (blockIdx.x / nb0) % nb1;
    const int bz = blockIdx.x / (nb0 * nb1);
    const int bs[3] = {bx * B16, by * B16, bz * B16};
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int rs = rec_start[blockIdx.x], nrec = rec_start[blockIdx.x + 1] - rs;
    const int nch = (nrec + kTcChunk - 1) / kTcChunk;
    const int nbt = (nrec + kTcKB - 1) / kTcKB;  // batches
    auto chunk_copy = [&](int c) {               // thread 0 only
        const int n = nrec - c * kTcChunk < kTcChunk ? nrec - c * kTcChunk : kTcChunk;
        tc::bulk_g2s(T.pts[c & 1], rec + (int64_t)(rs + c * kTcChunk) * R, (uint32_t)(n * R * 4), &T.cpbar[c & 1]);
    };
    int cp_issued = 0;  // bulk copies issued (thread 0)
    if (tid == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&T.full[i], kTcBuilderWarps);
            tc::mbar_init(&T.empty[i], 1);
            tc::mbar_init(&T.cpbar[i], 1);
        }
        tc::fence_mbar_init();
        T.fail = 0;
        for (; cp_issued < 2 && cp_issued < nch; ++cp_issued) chunk_copy(cp_issued);
    }
    {  // zero operands A (float4 stores)
        float4* a4 = reinterpret_cast<float4*>(&T.A[0][0][0]);
        for (int i = tid; i < (int)(sizeof(T.A) / sizeof(float4)); i += kTcThreads) a4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (warp == 0) tc::tmem_alloc(&T.tslot, 128);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = T.tslot;
    auto give_up = [&]() {
        *fail = 1;
        atomicExch(status, 1);
    };
    if (warp == 0) {
        // ---- issuing thread ----
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_tf32(128, 48);
            int issued = 0;
            for (int b = 0; b < nbt; ++b) {
                const int st = b & 1;
                if (b > 0 && b % kTcBatchesPerChunk == 0) {
                    // batch b starts chunk c - 1; every batch of chunk c - 2 (the previous content of
                    // chunk c's buffer) has been written, so its records have been read
                    const int c = b / kTcBatchesPerChunk + 1;
                    if (c < nch) {
                        tc::fence_async_shared();
                        chunk_copy(c);
                        cp_issued = c + 1;
                    }
                }
                if (*fail || !tc::mbar_wait(&T.full[st], (b >> 1) & 1, kTcWaitLimit)) {
                    give_up();
                    break;
                }
                tc::fence_after_sync();
                constexpr uint32_t lbo = 128, sbo = 128 * (kTcKB / 4);
#pragma unroll
                for (int s = 0; s < kTcKB / 8; ++s) {
                    const uint64_t bh = tc::smem_desc(tc::smem_u32(T.B[st][0]) + 256 * s, lbo, sbo);
                    const uint64_t bl = tc::smem_desc(tc::smem_u32(T.B[st][1]) + 256 * s, lbo, sbo);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t a0 = tc::smem_u32(T.A[st][0]) + 8192 * h + 256 * s;
                        const uint32_t a1 = tc::smem_u32(T.A[st][1]) + 8192 * h + 256 * s;
                        const uint64_t ah = tc::smem_desc(a0, lbo, sbo);
                        const uint64_t al = tc::smem_desc(a1, lbo, sbo);
                        const uint32_t d = tmem + 64 * h;
                        tc::mma_tf32(d, ah, bh, idesc, (b == 0 && s == 0) ? 0u : 1u);
                        tc::mma_tf32(d, ah, bl, idesc, 1u);
                        tc::mma_tf32(d, al, bh, idesc, 1u);
                    }
                }
                tc::commit(&T.empty[st]);
                issued = b + 1;
            }
            // all multiplications done (the last commit covers every earlier one); after a failure,
            // also the bulk copies still in flight (copy c completes phase c / 2 of buffer c % 2)
            if (issued > 0 && !tc::mbar_wait(&T.empty[(issued - 1) & 1], ((issued - 1) >> 1) & 1, kTcWaitLimit)) {
                give_up();
                tc::mbar_wait(&T.empty[(issued - 1) & 1], ((issued - 1) >> 1) & 1, kTcWaitLimit);
            }
            if (*fail)
                for (int c = cp_issued - 2 < 0 ? 0 : cp_issued - 2; c < cp_issued; ++c)
                    tc::mbar_wait(&T.cpbar[c & 1], (c >> 1) & 1, kTcWaitLimit);
        }
        __syncwarp();
    } else {
        // ---- builders ----
        // A: W / 2 warps, W threads per point slot (slot = at / W, x entry ix = at % W; a slot may span
        // two warps).  Each thread keeps, per operand stage, the corner of the footprint its slot held
        // there, clears the entries of that footprint in its column that the new footprint does not
        // cover, and writes its column of the new footprint: no entry is both cleared and written, and
        // no thread reads another's, so the slot needs no synchronisation.  B: the other builder warps.
        constexpr int kAW = W / 2;
        const bool builds_a = warp <= kAW;
        const int at = tid - 32;
        const int aslot = at / W, ix = at % W;
        const int r8 = lane >> 2, kk = lane & 3;                  // B: row and K entry within a core matrix
        const int kof = (aslot >> 2) * 32 + (aslot & 3);          // A: K offset of the slot
        int hx0 = 64, hy0 = 64, hx1 = 64, hy1 = 64;              // footprint corner held per stage (64: none)
        int b = 0;
        for (int ch = 0; ch < nch; ++ch) {
            if (*fail || !tc::mbar_wait(&T.cpbar[ch & 1], (ch >> 1) & 1, kTcWaitLimit)) {
                give_up();
                break;
            }
            const float* pts = T.pts[ch & 1];
            const int np = nrec - ch * kTcChunk < kTcChunk ? nrec - ch * kTcChunk : kTcChunk;
            for (int p0 = 0; p0 < np; p0 += kTcKB, ++b) {
                const int st = b & 1;
                if (b >= 2 && (*fail || !tc::mbar_wait(&T.empty[st], ((b >> 1) - 1) & 1, kTcWaitLimit))) {
                    give_up();
                    break;
                }
                const int nb = np - p0 < kTcKB ? np - p0 : kTcKB;
                if (builds_a) {
                    float* Ah = T.A[st][0];
                    float* Al = T.A[st][1];
                    const int ox = st ? hx1 : hx0, oy = st ? hy1 : hy0;
                    int nx = 64, ny = 64;
                    const float* pt = pts + (p0 + aslot) * R;
                    if (aslot < nb) {
                        const int cpk = __float_as_int(pt[3]);
                        nx = (cpk & 255) - 64;
                        ny = ((cpk >> 8) & 255) - 64;
                    }
                    if (ox < 64) {  // clear the old footprint's entries outside the new one
                        const int x = ox + ix;
                        if ((unsigned)x < 16u) {
                            const int base = (x >> 3) * 128 + (x & 7) * 4 + kof;
                            const bool xin = (unsigned)(x - nx) < (unsigned)W;
#pragma unroll
                            for (int iy = 0; iy < W; ++iy) {
                                const int y = oy + iy;
                                if ((unsigned)y < 16u && !(xin && (unsigned)(y - ny) < (unsigned)W)) {
                                    Ah[256 * y + base] = 0.0f;
                                    Al[256 * y + base] = 0.0f;
                                }
                            }
                        }
                    }
                    if (aslot < nb) {  // write the new footprint's column
                        const int x = nx + ix;
                        if ((unsigned)x < 16u) {
                            const float fx = pt[4 + ix];
                            const int base = (x >> 3) * 128 + (x & 7) * 4 + kof;
#pragma unroll
                            for (int iy = 0; iy < W; ++iy) {
                                const int y = ny + iy;
                                if ((unsigned)y < 16u) {
                                    const float v = pt[4 + W + iy] * fx;
                                    const float hi = tc::to_tf32(v);
                                    Ah[256 * y + base] = hi;
                                    Al[256 * y + base] = tc::to_tf32(v - hi);
                                }
                            }
                        }
                    }
                    if (st) {
                        hx1 = nx;
                        hy1 = ny;
                    } else {
                        hx0 = nx;
                        hy0 = ny;
                    }
                } else {
                    // B (dense): q_c phi_z(z) for rows n = (c, z)
                    float* Bh = T.B[st][0];
                    float* Bl = T.B[st][1];
#pragma unroll 2
                    for (int cm = warp - 1 - kAW; cm < 6 * (kTcKB / 4); cm += kTcBuilderWarps - kAW) {
                        const int g = cm >> 2, kg = cm & 3;
                        const int n = 8 * g + r8, k = 4 * kg + kk;
                        const int c = n >> 4, z = n & 15;
                        float v = 0.0f;
                        if (k < nb) {
                            const float* pt = pts + (p0 + k) * R;
                            const int iz = z - (((__float_as_int(pt[3]) >> 16) & 255) - 64);
                            if ((unsigned)iz < (unsigned)W) v = pt[c] * pt[4 + 2 * W + iz];
                        }
                        const float hi = tc::to_tf32(v);
                        Bh[cm * 32 + lane] = hi;
                        Bl[cm * 32 + lane] = tc::to_tf32(v - hi);
                    }
                }
                tc::fence_async_shared();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&T.full[st]);
            }
            if (*fail) break;
        }
    }
    __syncthreads();
    tc::fence_after_sync();
    // ---- write the brick: warp w < 8 reads rows 32 (w % 4) .. + 31 of half w / 4; columns (c, z) ----
    if (warp < 8) {
        const int h = warp >> 2, qd = warp & 3;
        const int m = 32 * qd + lane;
        const int y = 8 * h + (m >> 4), x = m & 15;
        const bool have = nbt > 0 && !*fail;
        const int64_t ng = S.ngrid;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float v[16];
            if (have) {
                tc::tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + 64 * h + 16 * c, v);
            } else {
#pragma unroll
                for (int z = 0; z < 16; ++z) v[z] = 0.0f;
            }
#pragma unroll
            for (int z = 0; z < 16; ++z)
                grid[c * ng + ((int64_t)(bs[2] + z) * S.n[1] + (bs[1] + y)) * S.n[0] + bs[0] + x] = v[z];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

// Register-column brick spreading for 16^3 bricks (no atomics at all): the 256 threads of a CTA
// are the 16 x 16 (x, y) columns of the brick and each keeps its column's 16 z values of the
// three components in registers.  The points whose footprint meets the brick are staged in
// batches in shared memory as brick-aligned, zero-padded kernel rows phi_x[16], phi_y[16],
// phi_z[16], so every point is one unconditional rank-1 update per thread:
//     acc_c[z] += q_c phi_x[x] phi_y[y] * phi_z[z].
// A warp covers two y rows and skips the points whose footprint misses both.
constexpr int kColB = 16;
constexpr int kColThreads = 256;
constexpr int kColBatch = 32;

template <typename T>
struct ColSlot {
    T q[4];          // charges (q[3] unused)
    T px[kColB];     // brick-aligned kernel rows, zero outside the footprint
    T py[kColB];
    T pz[kColB];
};

template <typename T>
__global__ void __launch_bounds__(kColThreads, 2) spread_column_kernel(
    LRSizes S, int nb0, int nb1, int nb2, const int32_t* __restrict__ bin_start, const T* __restrict__ binned,
    const int32_t* __restrict__ foot, T* __restrict__ grid) {
    __shared__ __align__(16) ColSlot<T> slot[kColBatch];
    __shared__ int2 yrange[kColBatch];  // overlap rows [lo, hi) in y; (0, 0) when the overlap is empty
    __shared__ int nbin_start[8], nbin_base[9];
    const int w = 2 * S.m;
    const int stride = 3 + 3 * w;
    const int bx = blockIdx.x % nb0;
    const int by = (blockIdx.x / nb0) % nb1;
    const int bz = blockIdx.x / (nb0 * nb1);
    const int bs[3] = {bx * kColB, by * kColB, bz * kColB};
    const int tx = threadIdx.x & (kColB - 1), ty = threadIdx.x / kColB;
    const int y0 = 2 * (threadIdx.x >> 5);  // the warp's rows: y0, y0 + 1
    if (threadIdx.x < 8) {
        const int nbr = threadIdx.x;
        const int cx = (bx - (nbr & 1) + nb0) % nb0;
        const int cy = (by - ((nbr >> 1) & 1) + nb1) % nb1;
        const int cz = (bz - ((nbr >> 2) & 1) + nb2) % nb2;
        const int b = (cz * nb1 + cy) * nb0 + cx;
        nbin_start[nbr] = bin_start[b];
        nbin_base[nbr + 1] = bin_start[b + 1] - bin_start[b];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        nbin_base[0] = 0;
        for (int k = 1; k <= 8; ++k) nbin_base[k] += nbin_base[k - 1];
    }
    __syncthreads();
    const int ntot = nbin_base[8];
    T acc0[kColB], acc1[kColB], acc2[kColB];
#pragma unroll
    for (int z = 0; z < kColB; ++z) acc0[z] = acc1[z] = acc2[z] = (T)0;
    for (int k0 = 0; k0 < ntot; k0 += kColBatch) {
        // ---- stage: 8 threads per point slot ----
        {
            const int s = threadIdx.x >> 3, part = threadIdx.x & 7;
            const int k = k0 + s;
            ColSlot<T>& sl = slot[s];
            if (k < ntot) {
                int nb = 0;
#pragma unroll
                for (int i = 1; i < 8; ++i) nb += k >= nbin_base[i];
                const int64_t j = nbin_start[nb] + (k - nbin_base[nb]);
                int o[3];
                bool empty = false;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    o[d] = foot[3 * j + d] - bs[d];
                    if (o[d] >= kColB) o[d] -= S.n[d];
                    const int lo = o[d] < 0 ? 0 : o[d];
                    const int hi = o[d] + w < kColB ? o[d] + w : kColB;
                    empty = empty || lo >= hi;
                }
                const T* src = binned + j * stride;
                for (int e = part; e < 3 * kColB; e += 8) {
                    const int d = e / kColB, t = e % kColB, r = t - o[d];
                    const T v = (r >= 0 && r < w) ? src[3 + d * w + r] : (T)0;
                    (d == 0 ? sl.px : d == 1 ? sl.py : sl.pz)[t] = v;
                }
                if (part < 3) sl.q[part] = src[part];
                if (part == 3) {
                    const int lo = o[1] < 0 ? 0 : o[1];
                    const int hi = o[1] + w < kColB ? o[1] + w : kColB;
                    yrange[s] = empty ? make_int2(0, 0) : make_int2(lo, hi);
                }
            } else if (part == 0) {
                yrange[s] = make_int2(0, 0);
            }
        }
        __syncthreads();
        // ---- accumulate ----
        const int nbatch = ntot - k0 < kColBatch ? ntot - k0 : kColBatch;
        for (int s = 0; s < nbatch; ++s) {
            const int2 yr = yrange[s];
            if (y0 + 2 <= yr.x || y0 >= yr.y) continue;  // warp-uniform
            const ColSlot<T>& sl = slot[s];
            const T fxy = sl.px[tx] * sl.py[ty];
            const T c0 = sl.q[0] * fxy, c1 = sl.q[1] * fxy, c2 = sl.q[2] * fxy;
#pragma unroll
            for (int z = 0; z < kColB; ++z) {
                const T f = sl.pz[z];
                acc0[z] = fma(c0, f, acc0[z]);
                acc1[z] = fma(c1, f, acc1[z]);
                acc2[z] = fma(c2, f, acc2[z]);
            }
        }
        __syncthreads();
    }
    const int64_t ng = S.ngrid;
    const int64_t plane = (int64_t)S.n[1] * S.n[0];
    T* g = grid + ((int64_t)bs[2] * S.n[1] + bs[1] + ty) * S.n[0] + bs[0] + tx;
#pragma unroll
    for (int z = 0; z < kColB; ++z) {
        g[z * plane] = acc0[z];
        g[ng + z * plane] = acc1[z];
        g[2 * ng + z * plane] = acc2[z];
    }
}

// Type-2 interpolation, one warp per node (cell order when available).  The node's 3 x W
// kernel values and wrapped grid indices go to shared memory (strided over the lanes); then the lanes
// take the W^3 footprint points in x-fastest order (consecutive lanes read consecutive x),
// several independent gathers in flight per lane, and the warp reduces the three components.
template <int W, typename T>  // kernel width 2m (compile-time: the footprint loop is unrolled)
__global__ void __launch_bounds__(256) interp_warp_kernel(
    LRSizes S, int64_t Np, const int32_t* __restrict__ order, const double* __restrict__ nodes, double sx0,
    double sx1, double sx2, const T* __restrict__ grid, double* __restrict__ out) {
    __shared__ T phs[8][3][W];
    __shared__ int ixs[8][3][W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    if (t >= Np) return;  // warp-uniform
    const int64_t i = order ? order[t] : t;
    for (int e = lane; e < 3 * W; e += 32) {  // 3 W entries (up to 48): some lanes take two
        const int d = e / W, s = e % W;
        const double scale = d == 0 ? sx0 : (d == 1 ? sx1 : sx2);
        const double xh = (nodes[d * Np + i] * scale) / (2.0 * kPi / S.n[d]);
        const int i0 = (int)floor(xh) - S.m + 1;
        phs[warp][d][s] = (T)es_kernel_w<W>(xh - (i0 + s), S.beta, S.edge, S.kernel);
        // the start folded once by a modulo (any i0, also from a non-finite node), then i0w + s < 2n
        ixs[warp][d][s] = wrap1(wrapi(i0, S.n[d]) + s, S.n[d]);
    }
    __syncwarp();
    const int64_t ng = S.ngrid, n0 = S.n[0], n1 = S.n[1];
    T a0 = 0, a1 = 0, a2 = 0;
    constexpr int kIter = (W * W * W + 31) / 32;
#pragma unroll 4
    for (int k = 0; k < kIter; ++k) {
        const int l = lane + 32 * k;
        if (l < W * W * W) {
            const int sx = l % W, sy = (l / W) % W, sz = l / (W * W);
            const T f = phs[warp][0][sx] * phs[warp][1][sy] * phs[warp][2][sz];
            const int64_t g = ((int64_t)ixs[warp][2][sz] * n1 + ixs[warp][1][sy]) * n0 + ixs[warp][0][sx];
            a0 += f * grid[g];
            a1 += f * grid[ng + g];
            a2 += f * grid[2 * ng + g];
        }
    }
    double b0 = a0, b1 = a1, b2 = a2;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        b0 += __shfl_xor_sync(0xffffffffu, b0, o);
        b1 += __shfl_xor_sync(0xffffffffu, b1, o);
        b2 += __shfl_xor_sync(0xffffffffu, b2, o);
    }
    if (lane == 0) {
        out[i] += b0;
        out[Np + i] += b1;
        out[2 * Np + i] += b2;
    }
}

int check_fft(vpbs_handle* h, cufftResult r, const char* what) {
    if (r == CUFFT_SUCCESS) return 0;
    return set_error(h, VPBS_ERR_CUDA, std::string("cuFFT error in ") + what + " (code " + std::to_string((int)r) + ")");
}

}  // namespace

int longrange_init(vpbs_handle* h) {
    LRSizes& S = h->lr;
    const vpbs_params& P = h->P;
    for (int d = 0; d < 3; ++d) {
        S.Ns[d] = P.Ns[d];
        S.n[d] = vpbs_fft_size(P.Ns[d], P.sigma);
    }
    S.nkx = P.Ns[0] / 2 + 1;
    S.nxc = S.n[0] / 2 + 1;
    S.ngrid = (int64_t)S.n[0] * S.n[1] * S.n[2];
    S.ncgrid = (int64_t)S.nxc * S.n[1] * S.n[2];
    S.nmodes = (int64_t)S.nkx * S.Ns[1] * S.Ns[2];
    S.m = P.m;
    S.kernel = P.nufft_kernel;
    if (S.kernel == VPBS_NUFFT_KAISER_BESSEL) {
        // the NFFT literature's shape parameter pi m (2 - 1/sigma) (Potts & Steidl 2003), scaled by 0.995
        S.beta = 0.995 * kPi * P.m * (2.0 - 1.0 / P.sigma);
        S.edge = S.beta / std::sinh(S.beta);
    } else {
        S.beta = 0.97 * kPi * (1.0 - 1.0 / (2.0 * P.sigma)) * (2.0 * P.m);
        S.edge = std::exp(-S.beta);
    }
    // brick edge for atomic-free spreading: divides every grid size, >= kernel width, >= 2 bricks
    h->gatherB = 0;
    for (int B : {16, 12, 10, 8}) {
        bool ok = B >= 2 * S.m;
        for (int d = 0; d < 3; ++d) ok = ok && S.n[d] % B == 0 && S.n[d] / B >= 2;
        if (ok) {
            h->gatherB = B;
            for (int d = 0; d < 3; ++d) h->nbrick[d] = S.n[d] / B;
            break;
        }
    }
    int rc;
    const bool mixed = P.precision == VPBS_PRECISION_MIXED;
    const size_t rsz = mixed ? sizeof(float) : sizeof(double);  // grid precision
    if ((rc = ensure(h, h->grid_r, rsz * 3 * S.ngrid, "real grid"))) return rc;
    if ((rc = ensure(h, h->grid_c, 2 * rsz * 3 * S.ncgrid, "complex grid"))) return rc;
    if ((rc = ensure(h, h->grid_c2, 2 * rsz * 3 * S.ncgrid, "complex grid (streamfunction)"))) return rc;
    if ((rc = ensure(h, h->uhat, sizeof(double2) * 3 * S.nmodes, "uhat"))) return rc;
    // separable deconvolution factors 1/psi_hat and 1/psi_hat * exp(-k^2 / 4 alpha^2) (the
    // Kaiser-Bessel filter is not separable: the Fourier kernel applies it per mode)
    std::vector<double> tab[6];
    const bool kb = P.splitting == VPBS_SPLITTING_KAISER_BESSEL;
    const double beta_g = kb ? 0.0 : -1.0 / (4.0 * P.alpha * P.alpha);
    for (int d = 0; d < 3; ++d) {
        const int len = d == 0 ? S.nkx : S.Ns[d];
        tab[d].resize(len);
        tab[3 + d].resize(len);
        const double k0 = 2.0 * kPi / P.L[d];
        for (int i = 0; i < len; ++i) {
            const int k = d == 0 ? i : mode_of(i, S.Ns[d]);
            const double dec = 1.0 / es_hat(2.0 * kPi * k / S.n[d], S.m, S.beta, S.kernel);
            const double kk = k0 * k;
            tab[d][i] = dec;
            tab[3 + d][i] = dec * std::exp(beta_g * kk * kk);
        }
    }
    size_t tot = 0;
    for (int d = 0; d < 6; ++d) tot += tab[d].size();
    if ((rc = ensure(h, h->decx, sizeof(double) * tot, "deconvolution tables"))) return rc;
    std::vector<double> all;
    all.reserve(tot);
    for (int d = 0; d < 6; ++d) all.insert(all.end(), tab[d].begin(), tab[d].end());
    if ((rc = check_cuda(h, cudaMemcpy(h->decx.p, all.data(), sizeof(double) * tot, cudaMemcpyHostToDevice), "copy tables")))
        return rc;
    int nrev[3] = {S.n[2], S.n[1], S.n[0]};
    if ((rc = check_fft(h, cufftPlanMany(&h->plan_r2c, 3, nrev, nullptr, 1, (int)S.ngrid, nullptr, 1, (int)S.ncgrid,
                                         mixed ? CUFFT_R2C : CUFFT_D2Z, 3), "plan r2c")))
        return rc;
    if ((rc = check_fft(h, cufftPlanMany(&h->plan_c2r, 3, nrev, nullptr, 1, (int)S.ncgrid, nullptr, 1, (int)S.ngrid,
                                         mixed ? CUFFT_C2R : CUFFT_Z2D, 3), "plan c2r")))
        return rc;
    h->have_plans = true;
    return 0;
}

void longrange_free(vpbs_handle* h) {
    if (h->have_plans) {
        cufftDestroy(h->plan_r2c);
        cufftDestroy(h->plan_c2r);
        h->have_plans = false;
    }
}

namespace {
inline cufftResult exec_r2c(cufftHandle p, double* in, double2* out) {
    return cufftExecD2Z(p, in, (cufftDoubleComplex*)out);
}
inline cufftResult exec_r2c(cufftHandle p, float* in, float2* out) { return cufftExecR2C(p, in, (cufftComplex*)out); }
inline cufftResult exec_c2r(cufftHandle p, double2* in, double* out) {
    return cufftExecZ2D(p, (cufftDoubleComplex*)in, out);
}
inline cufftResult exec_c2r(cufftHandle p, float2* in, float* out) { return cufftExecC2R(p, (cufftComplex*)in, out); }
}  // namespace

// T: grid precision (double for the plain form, float for the mixed form).
template <typename T>
int longrange_compute_t(vpbs_handle* h, int fields) {
    using C = typename std::conditional<std::is_same<T, double>::value, double2, float2>::type;
    const LRSizes& S = h->lr;
    const vpbs_params& P = h->P;
    int rc;
    const double sx[3] = {2.0 * kPi / P.L[0], 2.0 * kPi / P.L[1], 2.0 * kPi / P.L[2]};
    T* grid = (T*)h->grid_r.p;
    C* gc = (C*)h->grid_c.p;
    C* gc2 = (C*)h->grid_c2.p;
    // sources: cell-sorted copy (SoA x,y,z,qx,qy,qz), built by build_cell_lists
    const double* src = (const double*)h->src_sorted.p;
    if (h->gatherB) {
        StageScope st(h, ST_SPREAD);
        const int B = h->gatherB, nb0 = h->nbrick[0], nb1 = h->nbrick[1], nb2 = h->nbrick[2];
        const int64_t nbins = (int64_t)nb0 * nb1 * nb2, Nq = h->Nq;
        // FP32 grids with narrow kernels (m <= 4) on 16^3 bricks: tensor cores, with their own per-brick
        // records instead of the bins below
        const bool use_tc = std::is_same<T, float>::value && B == kColB && S.m <= 4 && h->spread_mode == 0;
        if ((rc = ensure(h, h->spread_bin, sizeof(int32_t) * 2 * Nq, "spread bins"))) return rc;
        if ((rc = ensure(h, h->spread_counts, sizeof(int32_t) * nbins, "spread bin counts"))) return rc;
        if ((rc = ensure(h, h->spread_start, sizeof(int32_t) * (nbins + 1), "spread bin starts"))) return rc;
        const int stride = 3 + 6 * S.m;  // values per binned point
        if ((rc = ensure(h, h->binned, sizeof(T) * stride * Nq, "binned points"))) return rc;
        if ((rc = ensure(h, h->spread_foot, sizeof(int32_t) * 3 * Nq, "footprints"))) return rc;
        int32_t* bin = (int32_t*)h->spread_bin.p;
        int32_t* rank = bin + Nq;
        int32_t* counts = (int32_t*)h->spread_counts.p;
        int32_t* start = (int32_t*)h->spread_start.p;
        int32_t* foot = (int32_t*)h->spread_foot.p;
        if (!use_tc) {
            if ((rc = check_cuda(h, cudaMemsetAsync(counts, 0, sizeof(int32_t) * nbins, h->stream), "memset"))) return rc;
            spread_bin_count_kernel<<<grid_for(Nq, 256), 256, 0, h->stream>>>(S, B, nb0, nb1, nb2, Nq, src, sx[0],
                                                                               sx[1], sx[2], bin, rank, counts);
            h->launches++;
            if ((rc = exclusive_scan(h, counts, start, nbins, h->scan_tmp_lr))) return rc;
            spread_bin_scatter_kernel<T><<<grid_for(Nq, 128), 128, 0, h->stream>>>(S, Nq, src, sx[0], sx[1], sx[2],
                                                                                    bin, rank, start, (T*)h->binned.p,
                                                                                    foot);
            h->launches++;
        }
        const unsigned nblk = (unsigned)nbins;
        const T* bsrc = (const T*)h->binned.p;
        const size_t smem = sizeof(T) * 3 * B * (B * (B + 1) + 8);
        auto launch = [&](auto kern) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            kern<<<nblk, kBrickThreads, smem, h->stream>>>(S, nb0, nb1, nb2, start, bsrc, foot, grid);
        };
        // plane-owner kernel (FP32 grids only; the branch that calls it is never taken for T = double)
        auto launch_plane = [&](void (*kern)(LRSizes, int, int, int, const int32_t*, const float*, const int32_t*,
                                             float*), int P) {
            const size_t psmem = sizeof(float) * 3 * kPlaneB * kPlaneB * (P == 8 ? PlaneLayout<8>::RX : PlaneLayout<4>::RX);
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem);
            kern<<<nblk, kPlaneThreads, psmem, h->stream>>>(S, nb0, nb1, nb2, start, (const float*)bsrc, foot,
                                                           (float*)grid);
        };
        switch (B) {
            case kColB:
                // FP32 grids with narrow kernels (m <= 4): the plane-owner kernel (the 16-deep
                // register columns mostly multiply zeros there); wider kernels and FP64 grids use
                // the columns
                if (use_tc) {
                    // tensor cores: per-brick records, then the brick product in 3xTF32
                    if ((rc = ensure_status(h))) return rc;
                    const int R = tc_record_floats(2 * S.m);
                    if ((rc = ensure(h, h->tc_counts, sizeof(int32_t) * 2 * nbins, "record counts"))) return rc;
                    if ((rc = ensure(h, h->tc_start, sizeof(int32_t) * (nbins + 1), "record starts"))) return rc;
                    if ((rc = ensure(h, h->tc_rec, sizeof(float) * R * 8 * (size_t)Nq, "brick records"))) return rc;
                    int32_t* tcount = (int32_t*)h->tc_counts.p;
                    int32_t* tfill = tcount + nbins;
                    if ((rc = check_cuda(h, cudaMemsetAsync(tcount, 0, sizeof(int32_t) * 2 * nbins, h->stream), "memset")))
                        return rc;
                    tc_rec_count_kernel<<<grid_for(Nq, 256), 256, 0, h->stream>>>(S, nb0, nb1, nb2, Nq, src, sx[0], sx[1],
                                                                                   sx[2], tcount);
                    if ((rc = exclusive_scan(h, tcount, (int32_t*)h->tc_start.p, nbins, h->scan_tmp_lr))) return rc;
                    auto launch_tc = [&](auto wtag) {
                        constexpr int W = decltype(wtag)::value;
                        tc_rec_scatter_kernel<W><<<grid_for(Nq, 128), 128, 0, h->stream>>>(
                            S, nb0, nb1, nb2, Nq, src, sx[0], sx[1], sx[2], (const int32_t*)h->tc_start.p, tfill,
                            (float*)h->tc_rec.p);
                        const size_t tsmem = sizeof(TcSpreadSmem);
                        cudaFuncSetAttribute(spread_tc_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem);
                        spread_tc_kernel<W><<<nblk, kTcThreads, tsmem, h->stream>>>(
                            S, nb0, nb1, (const int32_t*)h->tc_start.p, (const float*)h->tc_rec.p, (float*)grid,
                            h->status_dev);
                    };
                    switch (S.m) {
                        case 1: launch_tc(std::integral_constant<int, 2>()); break;
                        case 2: launch_tc(std::integral_constant<int, 4>()); break;
                        case 3: launch_tc(std::integral_constant<int, 6>()); break;
                        default: launch_tc(std::integral_constant<int, 8>()); break;
                    }
                    h->launches += 2;
                } else if (std::is_same<T, float>::value && S.m <= 4)
                    launch_plane(S.m <= 2 ? spread_plane_kernel<4> : spread_plane_kernel<8>, S.m <= 2 ? 4 : 8);
                else
                    spread_column_kernel<T><<<nblk, kColThreads, 0, h->stream>>>(S, nb0, nb1, nb2, start, bsrc, foot,
                                                                                 grid);
                break;
            case 12: launch(spread_brick_kernel<12, T>); break;
            case 10: launch(spread_brick_kernel<10, T>); break;
            default: launch(spread_brick_kernel<8, T>); break;
        }
        h->launches++;
        if ((rc = check_cuda(h, cudaGetLastError(), "spread gather kernels"))) return rc;
    } else {
        StageScope st(h, ST_SPREAD);
        if ((rc = check_cuda(h, cudaMemsetAsync(grid, 0, sizeof(T) * 3 * S.ngrid, h->stream), "memset grid")))
            return rc;
        spread_kernel_atomic<T><<<grid_for(h->Nq, kSpreadBatch), 256, 0, h->stream>>>(S, h->Nq, src, sx[0], sx[1], sx[2],
                                                                                      grid);
        h->launches++;
        if ((rc = check_cuda(h, cudaGetLastError(), "spread kernel"))) return rc;
    }
    {
        StageScope st(h, ST_FFT_FORWARD);
        if ((rc = check_fft(h, cufftSetStream(h->plan_r2c, h->stream), "set stream"))) return rc;
        if ((rc = check_fft(h, exec_r2c(h->plan_r2c, grid, gc), "exec r2c"))) return rc;
    }
    double kmax = INFINITY;
    for (int d = 0; d < 3; ++d) kmax = fmin(kmax, 2.0 * kPi * ((P.Ns[d] - 1) / 2) / P.L[d]);
    const double pref = P.Gamma / (P.L[0] * P.L[1] * P.L[2]);
    const bool kb = P.splitting == VPBS_SPLITTING_KAISER_BESSEL;
    const double* t = (const double*)h->decx.p;
    const double* dec0 = t;
    const double* dec1 = dec0 + S.nkx;
    const double* dec2 = dec1 + S.Ns[1];
    const double* decE0 = dec2 + S.Ns[2];
    const double* decE1 = decE0 + S.nkx;
    const double* decE2 = decE1 + S.Ns[1];
    {
        StageScope st(h, ST_FOURIER);
        fourier_kernel<C><<<grid_for(S.ncgrid, 256), 256, 0, h->stream>>>(
            S, pref, sx[0], sx[1], sx[2], P.truncate_spherical, kmax * kmax, fields, kb ? P.kb_beta * P.kb_beta : 0.0,
            P.rcut * P.rcut, kb ? P.kb_beta / std::sinh(P.kb_beta) : 0.0, dec0, dec1, dec2, decE0, decE1,
            decE2, gc, gc2, (double2*)h->uhat.p, 1);
        h->launches++;
        h->have_uhat = true;
        if ((rc = check_cuda(h, cudaGetLastError(), "fourier kernel"))) return rc;
    }
    if ((rc = check_fft(h, cufftSetStream(h->plan_c2r, h->stream), "set stream"))) return rc;
    const int32_t* order = (const int32_t*)h->dst_order.p;
    for (int f = 0; f < 2; ++f) {
        const int field = f == 0 ? VPBS_STREAMFUNCTION : VPBS_VELOCITY;
        if (!(fields & field)) continue;
        C* in = field == VPBS_VELOCITY ? gc : gc2;
        double* out = (double*)(field == VPBS_VELOCITY ? h->vel.p : h->psi.p);
        {
            StageScope st(h, ST_FFT_INVERSE);
            if ((rc = check_fft(h, exec_c2r(h->plan_c2r, in, grid), "exec c2r"))) return rc;
        }
        if (h->interp_wait) {
            if ((rc = check_cuda(h, cudaStreamWaitEvent(h->stream, h->interp_wait, 0), "wait short range"))) return rc;
        }
        StageScope st(h, ST_INTERP);
        auto launch_interp = [&](auto kern) {
            kern<<<grid_for(h->Np, 8), 256, 0, h->stream>>>(S, h->Np, order, (const double*)h->nodes.p, sx[0], sx[1],
                                                            sx[2], grid, out);
        };
        switch (S.m) {
            case 1: launch_interp(interp_warp_kernel<2, T>); break;
            case 2: launch_interp(interp_warp_kernel<4, T>); break;
            case 3: launch_interp(interp_warp_kernel<6, T>); break;
            case 4: launch_interp(interp_warp_kernel<8, T>); break;
            case 5: launch_interp(interp_warp_kernel<10, T>); break;
            case 6: launch_interp(interp_warp_kernel<12, T>); break;
            case 7: launch_interp(interp_warp_kernel<14, T>); break;
            default: launch_interp(interp_warp_kernel<16, T>); break;
        }
        h->launches++;
        if ((rc = check_cuda(h, cudaGetLastError(), "interp kernel"))) return rc;
    }
    return 0;
}

// interpolate_to_physical! with the default callback (longrange.jl:360-378): the field the
// reference's cache holds -- quantity 1: the (possibly coarse-grained) vorticity w_k as stored,
// 2: the streamfunction w_k / k^2, 3: the velocity i k x w_k / k^2 (both 0 at k = 0) -- times the
// type-2 deconvolution, written into the padded complex grid (no Ewald filter).
template <typename C>
__global__ void __launch_bounds__(256) field_grid_kernel(LRSizes S, double k0x, double k0y, double k0z, int quantity,
                                                        const double* __restrict__ dec0, const double* __restrict__ dec1,
                                                        const double* __restrict__ dec2,
                                                        const double2* __restrict__ uhat, C* __restrict__ gc) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= S.ncgrid) return;
    const int ix = (int)(idx % S.nxc);
    const int64_t rest = idx / S.nxc;
    const int iy = (int)(rest % S.n[1]);
    const int iz = (int)(rest / S.n[1]);
    const int ky = iy < (S.n[1] + 1) / 2 ? iy : iy - S.n[1];
    const int kz = iz < (S.n[2] + 1) / 2 ? iz : iz - S.n[2];
    const int lo1 = -(S.Ns[1] / 2), hi1 = (S.Ns[1] - 1) / 2;
    const int lo2 = -(S.Ns[2] / 2), hi2 = (S.Ns[2] - 1) / 2;
    const int64_t cstride = S.ncgrid;
    double2 r[3] = {{0, 0}, {0, 0}, {0, 0}};
    if (ix < S.nkx && ky >= lo1 && ky <= hi1 && kz >= lo2 && kz <= hi2) {
        const int ry = ky < 0 ? ky + S.Ns[1] : ky;
        const int rz = kz < 0 ? kz + S.Ns[2] : kz;
        const int64_t u = ((int64_t)rz * S.Ns[1] + ry) * S.nkx + ix;
        const double2 w0 = uhat[u], w1 = uhat[S.nmodes + u], w2 = uhat[2 * S.nmodes + u];
        const double kx = k0x * ix, kyy = k0y * ky, kzz = k0z * kz;
        const double k2 = kx * kx + kyy * kyy + kzz * kzz;
        const double k2inv = k2 == 0.0 ? 0.0 : 1.0 / k2;
        const double f = dec0[ix] * dec1[ry] * dec2[rz];
        if (quantity == 1) {
            r[0] = w0;
            r[1] = w1;
            r[2] = w2;
        } else if (quantity == 2) {
            r[0] = make_double2(w0.x * k2inv, w0.y * k2inv);
            r[1] = make_double2(w1.x * k2inv, w1.y * k2inv);
            r[2] = make_double2(w2.x * k2inv, w2.y * k2inv);
        } else {
            // i k x w / k^2 ; (i w).x = -w.y, (i w).y = w.x
            r[0] = make_double2(-(kyy * w2.y - kzz * w1.y) * k2inv, (kyy * w2.x - kzz * w1.x) * k2inv);
            r[1] = make_double2(-(kzz * w0.y - kx * w2.y) * k2inv, (kzz * w0.x - kx * w2.x) * k2inv);
            r[2] = make_double2(-(kx * w1.y - kyy * w0.y) * k2inv, (kx * w1.x - kyy * w0.x) * k2inv);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) r[c] = make_double2(r[c].x * f, r[c].y * f);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) gc[c * cstride + idx] = mkc<C>(r[c].x, r[c].y);
}

template <typename T>
int longrange_interpolate_t(vpbs_handle* h, int quantity, double* out) {
    using C = typename std::conditional<std::is_same<T, double>::value, double2, float2>::type;
    const LRSizes& S = h->lr;
    const vpbs_params& P = h->P;
    int rc;
    const double sx[3] = {2.0 * kPi / P.L[0], 2.0 * kPi / P.L[1], 2.0 * kPi / P.L[2]};
    T* grid = (T*)h->grid_r.p;
    C* gc = (C*)h->grid_c.p;
    const double* dec0 = (const double*)h->decx.p;
    const double* dec1 = dec0 + S.nkx;
    const double* dec2 = dec1 + S.Ns[1];
    field_grid_kernel<C><<<grid_for(S.ncgrid, 256), 256, 0, h->stream>>>(S, sx[0], sx[1], sx[2], quantity, dec0, dec1,
                                                                         dec2, (const double2*)h->uhat.p, gc);
    h->launches++;
    if ((rc = check_cuda(h, cudaGetLastError(), "field grid kernel"))) return rc;
    if ((rc = check_fft(h, cufftSetStream(h->plan_c2r, h->stream), "set stream"))) return rc;
    if ((rc = check_fft(h, exec_c2r(h->plan_c2r, gc, grid), "exec c2r"))) return rc;
    if ((rc = check_cuda(h, cudaMemsetAsync(out, 0, sizeof(double) * 3 * h->Np, h->stream), "memset"))) return rc;
    const int32_t* order = (const int32_t*)h->dst_order.p;
    auto launch_interp = [&](auto kern) {
        kern<<<grid_for(h->Np, 8), 256, 0, h->stream>>>(S, h->Np, order, (const double*)h->nodes.p, sx[0], sx[1], sx[2],
                                                        grid, out);
    };
    switch (S.m) {
        case 1: launch_interp(interp_warp_kernel<2, T>); break;
        case 2: launch_interp(interp_warp_kernel<4, T>); break;
        case 3: launch_interp(interp_warp_kernel<6, T>); break;
        case 4: launch_interp(interp_warp_kernel<8, T>); break;
        case 5: launch_interp(interp_warp_kernel<10, T>); break;
        case 6: launch_interp(interp_warp_kernel<12, T>); break;
        case 7: launch_interp(interp_warp_kernel<14, T>); break;
        default: launch_interp(interp_warp_kernel<16, T>); break;
    }
    h->launches++;
    return check_cuda(h, cudaGetLastError(), "interp kernel");
}

int longrange_compute(vpbs_handle* h, int fields) {
    return h->P.precision == VPBS_PRECISION_MIXED ? longrange_compute_t<float>(h, fields)
                                                  : longrange_compute_t<double>(h, fields);
}

}  // namespace vpbs

using namespace vpbs;

extern "C" int vpbs_interpolate_field(vpbs_handle* h, int32_t quantity, double* out_xyz) {
    if (!h || !out_xyz) return VPBS_ERR_ARG;
    if (quantity < 1 || quantity > 3)
        return set_error(h, VPBS_ERR_ARG, "quantity must be 1 (vorticity), 2 (streamfunction) or 3 (velocity)");
    if (!h->have_uhat || !h->have_points || h->Np == 0)
        return set_error(h, VPBS_ERR_STATE, "no long-range field: run a long-range computation first");
    int rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (rc) return rc;
    const int64_t Np = h->Np;
    double* d = nullptr;
    if ((rc = check_cuda(h, cudaMalloc(&d, sizeof(double) * 3 * Np), "cudaMalloc"))) return rc;
    rc = h->P.precision == VPBS_PRECISION_MIXED ? longrange_interpolate_t<float>(h, quantity, d)
                                                : longrange_interpolate_t<double>(h, quantity, d);
    std::vector<double> soa;
    if (!rc) {
        soa.resize((size_t)3 * Np);
        rc = check_cuda(h, cudaMemcpyAsync(soa.data(), d, sizeof(double) * 3 * Np, cudaMemcpyDeviceToHost, h->stream),
                        "D2H");
    }
    if (!rc) rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
    cudaFree(d);
    if (rc) return rc;
    for (int64_t i = 0; i < Np; ++i)
        for (int c = 0; c < 3; ++c) out_xyz[3 * i + c] = soa[(size_t)c * Np + i];
    return 0;
}

extern "C" int32_t vpbs_fft_size(int32_t Ns, double sigma) {
    int n = (int)std::ceil(sigma * Ns - 1e-9);
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
