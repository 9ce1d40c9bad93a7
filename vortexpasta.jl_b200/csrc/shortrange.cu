// Short-range part of the Ewald split on the device:
//  * local (LIA) term and self-interaction removal, one thread per node
//    (src/BiotSavart/shortrange/local_integrals.jl:4-165);
//  * cell lists as a counting sort of the quadrature points (and of the nodes) by cell
//    (replaces the linked lists of src/CellLists/gpu.jl:28-61 and the destination sort of
//    gpu.jl:183-231);
//  * the pair kernel (src/BiotSavart/shortrange/shortrange.jl:216-273 with the Gaussian
//    weights of splitting/gaussian.jl:273-279): one warp per destination node, lanes
//    stride over the contiguous cell-sorted source ranges of the (2M+1)^2 neighbour rows,
//    warp-shuffle reduction at the end.
#include <cmath>
#include <cstring>
#include <vector>

#include "vpbs_internal.cuh"
#include "periodic.cuh"

namespace vpbs {

// Interval and local coordinate of x in the FP32 cubic tables: k = floor(32 x) (rounded through
// the 1.5 * 2^23 trick, no conversion instruction), t = 32 x - k; k is clamped into [0, nf).
__host__ __device__ __forceinline__ void f32_table_pos(float x, int nf, int* k, float* t) {
    const float u = fmaf(x, kTabCInvH, -0.5f);
#if defined(__CUDA_ARCH__)
    const float y = __fadd_rn(u, 12582912.0f);
    const float kf = __fsub_rn(y, 12582912.0f);
    int kk = __float_as_int(y) - 0x4B400000;
#else
    volatile float yv = u + 12582912.0f;
    const float y = yv;
    volatile float kv = y - 12582912.0f;
    const float kf = kv;
    int kk;
    std::memcpy(&kk, &y, sizeof(int));
    kk -= 0x4B400000;
#endif
    *t = fmaf(x, kTabCInvH, -kf);
    const unsigned top = (unsigned)(nf - 1);
    *k = (int)((unsigned)kk < top ? (unsigned)kk : top);
}

__host__ __device__ __forceinline__ float f32_cubic(float4 c, float t) {
    return fmaf(fmaf(fmaf(c.w, t, c.z), t, c.y), t, c.x);
}

namespace {

__device__ __forceinline__ int64_t cell_of(const CellGrid& cg, const KParams& K, double x, double y, double z) {
    return cell_index(cg.nc, K.L, x, y, z);
}

// Cell of every element and its rank within the cell (atomic counter).
__global__ void cell_count_kernel(KParams K, CellGrid cg, int64_t n, const double* __restrict__ xyz,
                                  int32_t* __restrict__ cell, int32_t* __restrict__ rank,
                                  int32_t* __restrict__ counts) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int64_t c = cell_of(cg, K, xyz[j], xyz[n + j], xyz[2 * n + j]);
    cell[j] = (int32_t)c;
    rank[j] = warp_aggregated_rank(counts, (int32_t)c);
}

// Exclusive scan of counts[0..n) into start[0..n] with one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) scan_kernel(const int32_t* __restrict__ counts, int32_t* __restrict__ start,
                                                    int64_t n) {
    __shared__ int32_t part[1024];
    const int tid = threadIdx.x;
    const int64_t chunk = (n + 1023) / 1024;
    const int64_t lo = tid * chunk;
    const int64_t hi = lo + chunk < n ? lo + chunk : n;
    int32_t s = 0;
    for (int64_t i = lo; i < hi; ++i) s += counts[i];
    part[tid] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        int32_t v = tid >= off ? part[tid - off] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int32_t acc = part[tid] - s;  // exclusive prefix of this chunk
    for (int64_t i = lo; i < hi; ++i) {
        start[i] = acc;
        acc += counts[i];
    }
    if (tid == 1023) start[n] = part[1023];
}

// Multi-CTA exclusive scan for long count arrays: per-chunk sums, a scan of the sums (with
// scan_kernel), then every chunk scanned in shared memory from its offset.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanChunk = kScanThreads * kScanPer;

__device__ __forceinline__ int warp_incl_scan(int x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    return x;
}

__global__ void __launch_bounds__(kScanThreads) scan_partials_kernel(const int32_t* __restrict__ counts, int64_t n,
                                                                    int32_t* __restrict__ part) {
    __shared__ int wt[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanPer;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k)
        if (base + k < n) s += counts[base + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) wt[warp] = s;
    __syncthreads();
    if (warp == 0) {
        int v = wt[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) part[blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_chunks_kernel(const int32_t* __restrict__ counts, int64_t n,
                                                                  const int32_t* __restrict__ part_start,
                                                                  int32_t* __restrict__ start) {
    __shared__ int wt[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanPer;
    int c[kScanPer], s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        c[k] = base + k < n ? counts[base + k] : 0;
        s += c[k];
    }
    const int x = warp_incl_scan(s, lane);
    if (lane == 31) wt[warp] = x;
    __syncthreads();
    if (warp == 0) wt[lane] = warp_incl_scan(wt[lane], lane);
    __syncthreads();
    int acc = part_start[blockIdx.x] + (warp > 0 ? wt[warp - 1] : 0) + x - s;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (base + k < n) start[base + k] = acc;
        acc += c[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) start[n] = part_start[gridDim.x];
}

// Scatter the sources into cell order (SoA: x, y, z, qx, qy, qz) and record their segment.
__global__ void scatter_sources_kernel(int64_t Nq, int nquad, const double* __restrict__ points,
                                       const double* __restrict__ charges, const int32_t* __restrict__ cell,
                                       const int32_t* __restrict__ rank, const int32_t* __restrict__ start,
                                       double* __restrict__ sorted, int32_t* __restrict__ seg) {
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Nq) return;
    int64_t pos = (int64_t)start[cell[j]] + rank[j];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sorted[d * Nq + pos] = points[d * Nq + j];
        sorted[(3 + d) * Nq + pos] = charges[d * Nq + j];
    }
    seg[pos] = (int32_t)(j / nquad);
}

__global__ void scatter_nodes_kernel(int64_t Np, const int32_t* __restrict__ cell, const int32_t* __restrict__ rank,
                                     const int32_t* __restrict__ start, int32_t* __restrict__ order) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Np) return;
    order[(int64_t)start[cell[i]] + rank[i]] = (int32_t)i;
}

// Per-lane accumulators in the evaluation precision R; in FP32 they are Kahan-compensated
// (c holds the running compensation), in FP64 plain sums.
template <typename R>
struct PairAcc {
    R v[3], p[3];
    R cv[3], cp[3];
    unsigned long long inr, cand;
};

template <typename R>
__device__ __forceinline__ void acc_add(R& s, R& c, R x) {
    if constexpr (std::is_same<R, float>::value) {
        const R y = x - c;
        const R t = s + y;
        c = (t - s) - y;
        s = t;
    } else {
        s += x;
    }
}

__device__ __forceinline__ void ewald_weights_f(const KParams& K, float x, float& a, float& g) {
    int k = (int)(x * (float)kEwaldInvH);
    k = k < K.ewald_ntab ? k : K.ewald_ntab - 1;
    const float t = x - (k + 0.5f) * (float)kEwaldH;
    const float* ce = K.ewald_tab_f + k * kEwaldNCf;
    const float* cg = K.ewald_tab_f + (K.ewald_ntab + k) * kEwaldNCf;
    a = __ldg(ce + kEwaldNCf - 1);
    g = __ldg(cg + kEwaldNCf - 1);
#pragma unroll
    for (int n = kEwaldNCf - 2; n >= 0; --n) {
        a = fmaf(a, t, __ldg(ce + n));
        g = fmaf(g, t, __ldg(cg + n));
    }
}

// Per-warp queue of in-range pairs: the separations and source indices of candidates that
// passed the r^2 <= r_cut^2 test are compacted here (ballot + prefix popcount), so that the
// erfc/exp evaluation always runs on 32 live lanes instead of on the ~30% of lanes whose
// candidate happened to be in range.
constexpr int kPairThreads = 256;
constexpr int kQueue = 64;
struct PairQueue {
    double r[3][kQueue];
    int32_t j[kQueue];
};

// Pair integrand of entry k of the queue (short_range_integrand, integrands.jl:2-18).  R is
// the evaluation precision: the separation was formed in FP64 and is cast to R here.
template <bool VEL, bool PSI, typename R>
__device__ __forceinline__ void pair_eval(const KParams& K, const double* __restrict__ src, int64_t Ns,
                                          const PairQueue& Q, int k, PairAcc<R>& acc) {
    const R r0 = (R)Q.r[0][k], r1 = (R)Q.r[1][k], r2 = (R)Q.r[2][k];
    const int64_t j = Q.j[k];
    const R q0 = (R)src[3 * Ns + j], q1 = (R)src[4 * Ns + j], q2 = (R)src[5 * Ns + j];
    R rinv, wa = 1, wg = 1;  // erfc(alpha r) and erfc(alpha r) + 2/sqrt(pi) alpha r exp(-(alpha r)^2)
    if constexpr (std::is_same<R, float>::value) {
        rinv = rsqrtf(r0 * r0 + r1 * r1 + r2 * r2);
        if (K.ewald_ntab > 0) ewald_weights_f(K, (float)K.alpha / rinv, wa, wg);
    } else {
        const double r = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
        rinv = 1.0 / r;
        if (K.ewald_ntab > 0) ewald_weights(K, K.alpha * r, wa, wg);
    }
    if (VEL) {
        const R f = wg * rinv * rinv * rinv;
        acc_add<R>(acc.v[0], acc.cv[0], f * (q1 * r2 - q2 * r1));
        acc_add<R>(acc.v[1], acc.cv[1], f * (q2 * r0 - q0 * r2));
        acc_add<R>(acc.v[2], acc.cv[2], f * (q0 * r1 - q1 * r0));
    }
    if (PSI) {
        const R f = wa * rinv;
        acc_add<R>(acc.p[0], acc.cp[0], f * q0);
        acc_add<R>(acc.p[1], acc.cp[1], f * q1);
        acc_add<R>(acc.p[2], acc.cp[2], f * q2);
    }
}

template <bool VEL, bool PSI, typename R>
__device__ __forceinline__ void pair_range_q(const KParams& K, const double x[3], int64_t i, int32_t iprev,
                                             bool skip_local, const double* __restrict__ src, int64_t Ns,
                                             const int32_t* __restrict__ seg, int64_t b, int64_t e, int lane,
                                             PairAcc<R>& acc, PairQueue& Q, int& qcount) {
    for (int64_t base = b; base < e; base += 32) {
        const int64_t j = base + lane;
        bool inr = false;
        double r0 = 0, r1 = 0, r2 = 0;
        if (j < e && !(skip_local && (seg[j] == i || seg[j] == iprev))) {
            r0 = deper(x[0] - src[j], K.L[0], K.Lh[0], K.open_domain);
            r1 = deper(x[1] - src[Ns + j], K.L[1], K.Lh[1], K.open_domain);
            r2 = deper(x[2] - src[2 * Ns + j], K.L[2], K.Lh[2], K.open_domain);
            acc.cand++;
            inr = r0 * r0 + r1 * r1 + r2 * r2 <= K.rcut2;
        }
        const unsigned m = __ballot_sync(0xffffffffu, inr);
        if (inr) {
            const int pos = qcount + __popc(m & ((1u << lane) - 1u));
            Q.r[0][pos] = r0;
            Q.r[1][pos] = r1;
            Q.r[2][pos] = r2;
            Q.j[pos] = (int32_t)j;
            acc.inr++;
        }
        qcount += __popc(m);
        __syncwarp();
        if (qcount >= 32) {
            pair_eval<VEL, PSI, R>(K, src, Ns, Q, lane, acc);
            __syncwarp();
            const int rest = qcount - 32;
            if (lane < rest) {
                Q.r[0][lane] = Q.r[0][32 + lane];
                Q.r[1][lane] = Q.r[1][32 + lane];
                Q.r[2][lane] = Q.r[2][32 + lane];
                Q.j[lane] = Q.j[32 + lane];
            }
            __syncwarp();
            qcount = rest;
        }
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One warp per destination node (visited in cell order when cell lists are used).  R = double
// for the plain form, float for the mixed form (separations always formed in FP64).
template <bool VEL, bool PSI, typename R>
__global__ void __launch_bounds__(256) pair_kernel(
    KParams K, CellGrid cg, int64_t Np, int64_t Ns, const int32_t* __restrict__ dst_order,
    const double* __restrict__ nodes, const int32_t* __restrict__ idx_prev, const double* __restrict__ src,
    const int32_t* __restrict__ src_start, const int32_t* __restrict__ seg, int use_cells, int skip_local,
    double* __restrict__ vel, double* __restrict__ psi, unsigned long long* __restrict__ counters) {
    __shared__ PairQueue queues[kPairThreads / 32];
    const int lane = threadIdx.x & 31;
    const int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= Np) return;
    PairQueue& Q = queues[threadIdx.x >> 5];
    int qcount = 0;
    const int64_t i = use_cells ? dst_order[w] : w;
    const double x[3] = {nodes[i], nodes[Np + i], nodes[2 * Np + i]};
    const int32_t iprev = idx_prev[i];
    PairAcc<R> acc = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0ull, 0ull};
    if (!use_cells) {
        pair_range_q<VEL, PSI, R>(K, x, i, iprev, skip_local, src, Ns, seg, 0, Ns, lane, acc, Q, qcount);
    } else {
        const int M = cg.M;
        const int nc0 = cg.nc[0], nc1 = cg.nc[1], nc2 = cg.nc[2];
        const int cx = cell_coord(x[0], K.L[0], nc0);
        const int cy = cell_coord(x[1], K.L[1], nc1);
        const int cz = cell_coord(x[2], K.L[2], nc2);
        for (int dz = -M; dz <= M; ++dz) {
            int zz = cz + dz;
            zz = zz < 0 ? zz + nc2 : (zz >= nc2 ? zz - nc2 : zz);
            for (int dy = -M; dy <= M; ++dy) {
                int yy = cy + dy;
                yy = yy < 0 ? yy + nc1 : (yy >= nc1 ? yy - nc1 : yy);
                const int64_t base = ((int64_t)zz * nc1 + yy) * nc0;
                const int lo = cx - M * cg.G, hi = cx + M * cg.G;  // M cells = M G slabs in x
                if (lo >= 0 && hi < nc0) {
                    pair_range_q<VEL, PSI, R>(K, x, i, iprev, skip_local, src, Ns, seg, src_start[base + lo],
                                         src_start[base + hi + 1], lane, acc, Q, qcount);
                } else if (lo < 0) {
                    pair_range_q<VEL, PSI, R>(K, x, i, iprev, skip_local, src, Ns, seg, src_start[base + lo + nc0],
                                         src_start[base + nc0], lane, acc, Q, qcount);
                    pair_range_q<VEL, PSI, R>(K, x, i, iprev, skip_local, src, Ns, seg, src_start[base],
                                         src_start[base + hi + 1], lane, acc, Q, qcount);
                } else {
                    pair_range_q<VEL, PSI, R>(K, x, i, iprev, skip_local, src, Ns, seg, src_start[base + lo],
                                         src_start[base + nc0], lane, acc, Q, qcount);
                    pair_range_q<VEL, PSI, R>(K, x, i, iprev, skip_local, src, Ns, seg, src_start[base],
                                         src_start[base + hi - nc0 + 1], lane, acc, Q, qcount);
                }
            }
        }
    }
    if (lane < qcount) pair_eval<VEL, PSI, R>(K, src, Ns, Q, lane, acc);  // queue remainder
    const double pref = K.Gamma / (4.0 * kPi);
    double v0 = 0, v1 = 0, v2 = 0, p0 = 0, p1 = 0, p2 = 0;
    // lane partial sums (compensated in FP32) are reduced across the warp in FP64
    auto lane_total = [](R s, R c) { return (double)s - (double)c; };
    if (VEL) {
        v0 = warp_sum(lane_total(acc.v[0], acc.cv[0]));
        v1 = warp_sum(lane_total(acc.v[1], acc.cv[1]));
        v2 = warp_sum(lane_total(acc.v[2], acc.cv[2]));
    }
    if (PSI) {
        p0 = warp_sum(lane_total(acc.p[0], acc.cp[0]));
        p1 = warp_sum(lane_total(acc.p[1], acc.cp[1]));
        p2 = warp_sum(lane_total(acc.p[2], acc.cp[2]));
    }
    unsigned long long inr = warp_sum_u(acc.inr), cand = warp_sum_u(acc.cand);
    if (lane == 0) {
        if (VEL) { vel[i] += pref * v0; vel[Np + i] += pref * v1; vel[2 * Np + i] += pref * v2; }
        if (PSI) { psi[i] += pref * p0; psi[Np + i] += pref * p1; psi[2 * Np + i] += pref * p2; }
        atomicAdd(&counters[0], inr);
        atomicAdd(&counters[1], cand);
    }
}

// ---- cell-tiled pair kernel ----
// One CTA per destination cell.  The sources of the (2M+1)^3 neighbour cells (in x: the G
// slabs of each) are concatenated in (row (dy, dz), slab) order and streamed through shared
// memory in tiles of kTile sources, as coordinates relative to the cell corner (already
// shifted to the periodic image next to the cell) split into FP32 hi + lo parts.  Per
// destination and row the candidate range is trimmed to the slabs within r_cut of the node.
// Candidates are screened on the hi parts in FP32 against r_cut^2 (1 + 2e-5) -- the FP32
// rounding of r^2 stays below 1e-6 r_cut^2 here, so no pair in range is lost -- and queued; the
// queued pairs are decided (r^2 <= r_cut^2) and evaluated with the separation formed in FP64
// from the hi + lo parts (relative error ~1e-15), two pairs per lane at a time so that their
// dependency chains overlap.  Destinations are handled in passes of up to kPassDst nodes;
// warps take (destination, row-part) items and add each item's warp-reduced sum to the
// destination's shared-memory accumulator.
constexpr int kTile = 2560;
constexpr int kTilePad = kTile + 32;  // a chunk of 32 lanes may read past the tile end (masked)
constexpr int kPassDst = 64;
constexpr int kMaxNbCells = 2048;  // neighbour slabs of a block: rows x slabs per row
constexpr int kMaxBlockRows = 16;  // (y, z) cell rows of a block (destination ranges)
constexpr int kMaxRows = 81;      // (2M+1)^2
constexpr int kTileQueue = 128;   // screened pairs are evaluated 64 at a time (two per lane)
constexpr double kScreenMargin = 2e-5;

struct TileSmem {
    // relative source position split as hi + lo FP32 parts (|lo| <= ulp(hi) / 2, together ~48
    // significant bits); hi.w holds the cell-sorted index, lo.w the segment (int bits)
    float4 hi[kTilePad];
    float4 lo[kTilePad];
    int32_t queue[kPairThreads / 32][kTileQueue];  // per warp: tile indices of screened pairs
    double acc[kPassDst][6];  // per destination: velocity, streamfunction
    double dx[kPassDst][3];   // destination positions
    int32_t di[kPassDst], dprev[kPassDst];
    int32_t dr_start[kMaxBlockRows], dr_base[kMaxBlockRows + 1];  // destination ranges of the block
    int32_t off[kMaxNbCells + 1];  // concatenated offsets of the neighbour slabs
    int32_t cstart[kMaxNbCells];   // first cell-sorted source of each neighbour slab
    int2 rng[kPairThreads / 32][kMaxRows];  // per warp: candidate range of every row
};

// 1/sqrt(s) in FP64: FP32 hardware estimate refined by two Newton-Raphson steps
// y <- y (3 - s y^2) / 2 (quadratic convergence: ~1e-7 -> ~1e-14 -> rounding level).
__device__ __forceinline__ double rsqrt_nr(double s) {
    double y = (double)rsqrtf((float)s);
    double t = s * y;
    y = y * fma(-0.5 * t, y, 1.5);
    t = s * y;
    y = y * fma(-0.5 * t, y, 1.5);
    return y;
}

// Both Ewald weights from the interleaved table (one 16-byte load per degree).
__device__ __forceinline__ void ewald_weights2(const KParams& K, double x, double& a, double& g) {
    int k = (int)(x * kEwaldInvH);
    k = k < K.ewald_ntab ? k : K.ewald_ntab - 1;
    const double t = x - (k + 0.5) * kEwaldH;
    const double2* c = K.ewald_tab2 + k * kEwaldNC;
    double2 v = __ldg(c + kEwaldNC - 1);
    a = v.x;
    g = v.y;
#pragma unroll
    for (int n = kEwaldNC - 2; n >= 0; --n) {
        v = __ldg(c + n);
        a = fma(a, t, v.x);
        g = fma(g, t, v.y);
    }
}

// One of the Ewald weights (erfc for the streamfunction, g for the velocity).
__device__ __forceinline__ double ewald_weight1(const KParams& K, double x, int which) {
    int k = (int)(x * kEwaldInvH);
    k = k < K.ewald_ntab ? k : K.ewald_ntab - 1;
    const double t = x - (k + 0.5) * kEwaldH;
    const double* c = K.ewald_tab + (which * K.ewald_ntab + k) * kEwaldNC;
    double a = __ldg(c + kEwaldNC - 1);
#pragma unroll
    for (int n = kEwaldNC - 2; n >= 0; --n) a = fma(a, t, __ldg(c + n));
    return a;
}

static_assert(sizeof(TileSmem) <= 113 * 1024, "two pair-kernel CTAs must fit in one SM's shared memory");

// Largest row r in [0, n] whose first concatenated index off[r W] is <= T (off[0] = 0 <= T).
__device__ __forceinline__ int last_row_le(const int32_t* off, int W, int n, int T) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid * W] <= T) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Distance from x to the cell [lo, lo + h], less a margin of 1e-9 h so that rounding in the
// binning can never cull a source that is in range.
__device__ __forceinline__ double box_gap(double x, double lo, double h) {
    const double g = fmax(fmax(lo - x, x - (lo + h)), 0.0);
    return fmax(g - 1e-9 * h, 0.0);
}

// Two queued pairs per lane (tile indices t0, t1; v0, v1 mark valid entries): the separation
// formed in FP64 from the hi + lo parts, the r^2 <= r_cut^2 decision, and the pair integrand
// (short_range_integrand, integrands.jl:2-18) in precision R.  Entries that are invalid or out
// of range are evaluated at a harmless separation (r_cut, 0, 0) with zero charge, so both
// chains run straight through.  Called by all lanes of the warp.
template <bool VEL, bool PSI, typename R>
__device__ __forceinline__ void tile_eval2(const KParams& K, const double xd[3], const TileSmem& S,
                                           const double* __restrict__ src, int64_t Ns, int t0, bool v0, int t1,
                                           bool v1, PairAcc<double>& acc, unsigned long long& ninr) {
    const int tt[2] = {t0, t1};
    const bool vv[2] = {v0, v1};
    double d[2][3], q[2][3], s2[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const float4 h = S.hi[tt[u]], l = S.lo[tt[u]];
        const int64_t j = __float_as_int(h.w);
#pragma unroll
        for (int c = 0; c < 3; ++c) q[u][c] = vv[u] ? src[(3 + c) * Ns + j] : 0.0;
        d[u][0] = xd[0] - ((double)h.x + (double)l.x);
        d[u][1] = xd[1] - ((double)h.y + (double)l.y);
        d[u][2] = xd[2] - ((double)h.z + (double)l.z);
        s2[u] = d[u][0] * d[u][0] + d[u][1] * d[u][1] + d[u][2] * d[u][2];
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const bool ok = vv[u] && s2[u] <= K.rcut2;
        ninr += __popc(__ballot_sync(0xffffffffu, ok));
        if (!ok) {
            d[u][0] = K.rcut;
            d[u][1] = d[u][2] = 0.0;
            s2[u] = K.rcut2;
            q[u][0] = q[u][1] = q[u][2] = 0.0;
        }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const R r0 = (R)d[u][0], r1 = (R)d[u][1], r2 = (R)d[u][2];
        R rinv, wa = 1, wg = 1;
        if constexpr (std::is_same<R, float>::value) {
            rinv = rsqrtf((float)s2[u]);
            ewald_weights_f(K, (float)K.alpha / rinv, wa, wg);
        } else {
            rinv = rsqrt_nr(s2[u]);
            const double xa = K.alpha * (s2[u] * rinv);
            if (VEL && PSI) ewald_weights2(K, xa, wa, wg);
            else if (VEL) wg = ewald_weight1(K, xa, 1);
            else wa = ewald_weight1(K, xa, 0);
        }
        // each pair's contribution is formed in R and accumulated in FP64
        const R q0 = (R)q[u][0], q1 = (R)q[u][1], q2 = (R)q[u][2];
        if (VEL) {
            const R f = wg * rinv * rinv * rinv;
            acc.v[0] += (double)(f * (q1 * r2 - q2 * r1));
            acc.v[1] += (double)(f * (q2 * r0 - q0 * r2));
            acc.v[2] += (double)(f * (q0 * r1 - q1 * r0));
        }
        if (PSI) {
            const R f = wa * rinv;
            acc.p[0] += (double)(f * q0);
            acc.p[1] += (double)(f * q1);
            acc.p[2] += (double)(f * q2);
        }
    }
}

// Candidates [a, b) of the tile against the destination (cell-relative position xd in FP64,
// xr in FP32; node i, previous node iprev): FP32 screen on the hi parts, compaction of the
// survivors into the warp's queue, evaluation 64 at a time.
template <bool VEL, bool PSI, bool SKIP, typename R>
__device__ __forceinline__ void tile_range_q(const KParams& K, const double xd[3], float3 xr, float rc2s, int i,
                                             int iprev, const TileSmem& S, const double* __restrict__ src, int64_t Ns,
                                             int a, int b, int lane, PairAcc<double>& acc, int32_t* Q, int& qcount,
                                             unsigned long long& ninr) {
    for (int base = a; base < b; base += 32) {
        const int t = base + lane;
        const float4 p = S.hi[t];
        const float e0 = xr.x - p.x, e1 = xr.y - p.y, e2 = xr.z - p.z;
        bool inr = t < b && fmaf(e0, e0, fmaf(e1, e1, e2 * e2)) <= rc2s;
        if (SKIP) {
            const int sg = __float_as_int(S.lo[t].w);
            inr = inr && sg != i && sg != iprev;
        }
        const unsigned m = __ballot_sync(0xffffffffu, inr);
        if (inr) Q[qcount + __popc(m & ((1u << lane) - 1u))] = t;
        qcount += __popc(m);
        __syncwarp();
        if (qcount >= 64) {
            tile_eval2<VEL, PSI, R>(K, xd, S, src, Ns, Q[lane], true, Q[32 + lane], true, acc, ninr);
            __syncwarp();
            if (lane < qcount - 64) Q[lane] = Q[64 + lane];
            __syncwarp();
            qcount -= 64;
        }
    }
}

template <bool VEL, bool PSI, bool SKIP, typename R>
__global__ void __launch_bounds__(kPairThreads, 2) pair_cell_kernel(
    KParams K, CellGrid cg, int64_t Np, int64_t Ns, const int32_t* __restrict__ dst_start,
    const int32_t* __restrict__ dst_order, const double* __restrict__ nodes, const int32_t* __restrict__ idx_prev,
    const double* __restrict__ src, const int32_t* __restrict__ src_start, const int32_t* __restrict__ seg,
    double* __restrict__ vel, double* __restrict__ psi, unsigned long long* __restrict__ counters, int3 bk,
    int3 nb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem& S = *reinterpret_cast<TileSmem*>(smem_raw);
    const int M = cg.M, G = cg.G;
    const int nc0 = cg.nc[0], nc1 = cg.nc[1], nc2 = cg.nc[2];
    const int ncc = nc0 / G;  // cells in x (each made of G slabs)
    // this CTA's block of cells [cx0, cx1) x [cy0, cy1) x [cz0, cz1)
    const int bxi = blockIdx.x % nb.x, byi = (blockIdx.x / nb.x) % nb.y, bzi = blockIdx.x / (nb.x * nb.y);
    const int cx0 = bxi * bk.x, cx1 = min(cx0 + bk.x, ncc);
    const int cy0 = byi * bk.y, cy1 = min(cy0 + bk.y, nc1);
    const int cz0 = bzi * bk.z, cz1 = min(cz0 + bk.z, nc2);
    const int ndr = (cy1 - cy0) * (cz1 - cz0);  // destination ranges: one per (y, z) cell row
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < ndr; ++k) {
            const int yy = cy0 + k % (cy1 - cy0), zz = cz0 + k / (cy1 - cy0);
            const int64_t s0 = ((int64_t)zz * nc1 + yy) * nc0 + (int64_t)cx0 * G;
            const int a = dst_start[s0], b = dst_start[s0 + (int64_t)(cx1 - cx0) * G];
            S.dr_start[k] = a;
            S.dr_base[k] = acc;
            acc += b - a;
        }
        S.dr_base[ndr] = acc;
    }
    __syncthreads();
    const int nd = S.dr_base[ndr];
    if (nd == 0) return;  // uniform over the CTA
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double hx = K.L[0] / nc0, h1 = K.L[1] / nc1, h2 = K.L[2] / nc2, inv_hx = nc0 / K.L[0];
    // neighbourhood: rows (y, z) of the block widened by M cells, slabs in x widened by M G
    const int WY = cy1 - cy0 + 2 * M, WZ = cz1 - cz0 + 2 * M, WX = (cx1 - cx0 + 2 * M) * G;
    const int nrow = WY * WZ, ncb = nrow * WX;
    const int ry0 = cy0 - M, rz0 = cz0 - M, xs0 = cx0 * G - M * G;  // unwrapped first row / slab
    const double o0 = cx0 * G * hx, o1 = cy0 * h1, o2 = cz0 * h2;  // block corner: origin of the FP32 coordinates
    const float rc2s = (float)(K.rcut2 * (1.0 + kScreenMargin));
    // neighbour slabs in (row, slab) order: first cell-sorted source and count
    for (int ci = threadIdx.x; ci < ncb; ci += kPairThreads) {
        const int r = ci / WX, k = ci % WX;
        int xx = xs0 + k, yy = ry0 + r % WY, zz = rz0 + r / WY;
        xx = xx < 0 ? xx + nc0 : (xx >= nc0 ? xx - nc0 : xx);
        yy = yy < 0 ? yy + nc1 : (yy >= nc1 ? yy - nc1 : yy);
        zz = zz < 0 ? zz + nc2 : (zz >= nc2 ? zz - nc2 : zz);
        const int64_t c = ((int64_t)zz * nc1 + yy) * nc0 + xx;
        const int s0 = src_start[c];
        S.cstart[ci] = s0;
        S.off[ci + 1] = src_start[c + 1] - s0;
    }
    __syncthreads();
    if (warp == 0) {  // counts -> concatenated offsets
        int carry = 0;
        for (int base = 0; base < ncb; base += 32) {
            const int ci = base + lane;
            int v = ci < ncb ? S.off[ci + 1] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            if (ci < ncb) S.off[ci + 1] = carry + v;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
        if (lane == 0) S.off[0] = 0;
    }
    __syncthreads();
    const int ntot = S.off[ncb];
    const double pref = K.Gamma / (4.0 * kPi);
    unsigned long long ninr = 0, ncand = 0;  // warp-uniform
    for (int p0 = 0; p0 < nd; p0 += kPassDst) {
        const int np = nd - p0 < kPassDst ? nd - p0 : kPassDst;
        __syncthreads();  // the previous pass has written its results
        for (int t = threadIdx.x; t < np; t += kPairThreads) {
            const int tt = p0 + t;
            int k = 0;
            while (k + 1 < ndr && S.dr_base[k + 1] <= tt) ++k;
            const int i = dst_order[S.dr_start[k] + tt - S.dr_base[k]];
            S.di[t] = i;
            S.dprev[t] = idx_prev[i];
#pragma unroll
            for (int d = 0; d < 3; ++d) S.dx[t][d] = nodes[d * Np + i];
#pragma unroll
            for (int c = 0; c < 6; ++c) S.acc[t][c] = 0.0;
        }
        const int P = np >= kPairThreads / 32 ? 1 : (kPairThreads / 32) / np;  // row parts per destination
        const int nitems = np * P;
        for (int T0 = 0, T1 = 0; T0 < ntot; T0 = T1) {
            // tile [T0, T1): whole rows [ra, rb) while they fit, else a kTile piece of one row
            const int ra = min(last_row_le(S.off, WX, nrow, T0), nrow - 1);
            const int rf = last_row_le(S.off, WX, nrow, T0 + kTile);
            T1 = S.off[rf * WX] > T0 ? S.off[rf * WX] : min(T0 + kTile, ntot);
            const int rb = min(last_row_le(S.off, WX, nrow, T1 - 1) + 1, nrow);
            __syncthreads();  // previous tile consumed, destinations loaded
            // staging, a warp per row (periodic image of each slab next to the destination block): the
            // slabs of a row are consecutive cells, so its sources are one contiguous range of the
            // cell-sorted arrays, or two where the row wraps around the period in x
            const int kw = xs0 < 0 ? -xs0 : (xs0 + WX > nc0 ? nc0 - xs0 : WX);  // first slab past the wrap
            const double sxA = xs0 < 0 ? -K.L[0] : 0.0, sxB = xs0 < 0 ? 0.0 : K.L[0];
            for (int r = ra + warp; r < rb; r += kPairThreads / 32) {
                const int rowA = S.off[r * WX], rowE = S.off[(r + 1) * WX];
                const int a = rowA > T0 ? rowA : T0, b = rowE < T1 ? rowE : T1;
                if (a >= b) continue;  // warp-uniform
                const int yu = ry0 + r % WY, zu = rz0 + r / WY;
                const double sy = yu < 0 ? -K.L[1] : (yu >= nc1 ? K.L[1] : 0.0);
                const double sz = zu < 0 ? -K.L[2] : (zu >= nc2 ? K.L[2] : 0.0);
                const int offB = S.off[r * WX + kw];
                const int gA = S.cstart[r * WX];
                const int gB = kw < WX ? S.cstart[r * WX + kw] : 0;
                for (int t = a + lane; t < b; t += 32) {
                    const bool inA = t < offB;
                    const int j = inA ? gA + (t - rowA) : gB + (t - offB);
                    const double sx = inA ? sxA : sxB;
                    const double u0 = src[j] + sx - o0, u1 = src[Ns + j] + sy - o1, u2 = src[2 * Ns + j] + sz - o2;
                    const float f0 = (float)u0, f1 = (float)u1, f2 = (float)u2;
                    S.hi[t - T0] = make_float4(f0, f1, f2, __int_as_float(j));
                    S.lo[t - T0] = make_float4((float)(u0 - f0), (float)(u1 - f1), (float)(u2 - f2),
                                               __int_as_float(SKIP ? seg[j] : 0));
                }
            }
            __syncthreads();
            for (int it = warp; it < nitems; it += kPairThreads / 32) {
                const int dl = it % np, part = it / np;
                const double x[3] = {S.dx[dl][0], S.dx[dl][1], S.dx[dl][2]};
                // candidate range of every row, trimmed to the slabs within r_cut of the node
                for (int r = ra + lane; r < rb; r += 32) {
                    const double gy = box_gap(x[1], (ry0 + r % WY) * h1, h1);
                    const double gz = box_gap(x[2], (rz0 + r / WY) * h2, h2);
                    const double gyz = gy * gy + gz * gz;
                    int a = 0, b = 0;
                    if (gyz <= K.rcut2) {
                        const double w = (double)sqrtf((float)(K.rcut2 - gyz)) * (1.0 + 1e-6) + 1e-9 * hx;
                        int klo = (int)floor((x[0] - w) * inv_hx) - xs0;
                        int khi = (int)floor((x[0] + w) * inv_hx) - xs0;
                        klo = klo < 0 ? 0 : klo;
                        khi = khi > WX - 1 ? WX - 1 : khi;
                        if (klo <= khi) {
                            a = S.off[r * WX + klo];
                            b = S.off[r * WX + khi + 1];
                        }
                    }
                    S.rng[warp][r] = make_int2(a, b);
                }
                __syncwarp();
                PairAcc<double> acc = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0ull, 0ull};
                int qcount = 0;
                int32_t* Q = S.queue[warp];
                const double xd[3] = {x[0] - o0, x[1] - o1, x[2] - o2};
                const float3 xr = make_float3((float)xd[0], (float)xd[1], (float)xd[2]);
                const int i = S.di[dl], iprev = S.dprev[dl];
                for (int r = ra + part; r < rb; r += P) {
                    const int2 ab = S.rng[warp][r];
                    const int a = ab.x > T0 ? ab.x : T0, b = ab.y < T1 ? ab.y : T1;
                    if (a < b) {
                        ncand += b - a;
                        tile_range_q<VEL, PSI, SKIP, R>(K, xd, xr, rc2s, i, iprev, S, src, Ns, a - T0, b - T0, lane, acc, Q,
                                                        qcount, ninr);
                    }
                }
                if (qcount > 0)  // warp-uniform
                    tile_eval2<VEL, PSI, R>(K, xd, S, src, Ns, lane < qcount ? Q[lane] : 0, lane < qcount,
                                            32 + lane < qcount ? Q[32 + lane] : 0, 32 + lane < qcount, acc, ninr);
                double s[6] = {0, 0, 0, 0, 0, 0};
                if (VEL)
#pragma unroll
                    for (int c = 0; c < 3; ++c) s[c] = warp_sum(acc.v[c]);
                if (PSI)
#pragma unroll
                    for (int c = 0; c < 3; ++c) s[3 + c] = warp_sum(acc.p[c]);
                if (lane == 0) {
                    if (VEL)
                        for (int c = 0; c < 3; ++c) atomicAdd(&S.acc[dl][c], s[c]);
                    if (PSI)
                        for (int c = 0; c < 3; ++c) atomicAdd(&S.acc[dl][3 + c], s[3 + c]);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < np; t += kPairThreads) {
            const int64_t i = S.di[t];
            if (VEL) {
                vel[i] += pref * S.acc[t][0];
                vel[Np + i] += pref * S.acc[t][1];
                vel[2 * Np + i] += pref * S.acc[t][2];
            }
            if (PSI) {
                psi[i] += pref * S.acc[t][3];
                psi[Np + i] += pref * S.acc[t][4];
                psi[2 * Np + i] += pref * S.acc[t][5];
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&counters[0], ninr);
        atomicAdd(&counters[1], ncand);
    }
}

// ---- FP32 pair kernel of the mixed form ----
// Same decomposition as pair_cell_kernel (CTA per block of cells, the block's neighbour slabs
// concatenated in (row, slab) order and streamed through shared memory in row-aligned tiles,
// per-node candidate ranges trimmed to the slabs within r_cut), with every per-pair operation in
// FP32 and every operand in shared memory:
//  * staging: source position relative to the block corner split into FP32 hi + lo parts (from
//    the FP64 position), FP32 charge, segment index; 32-source units spread over all warps;
//  * per node, only the (2M+1)^2 rows around its own cell are examined (a lane each), and only
//    the non-empty ones are walked;
//  * screen: hi parts only, against r_cut^2 (1 + 2e-5) (their rounding is below 1e-6 r_cut^2);
//  * separation of a queued pair: (x_hi - s_hi) + (x_lo - s_lo) -- the FP64 separation rounded
//    to FP32 within ~2 ulps (the hi difference is rounded relative to the separation itself);
//  * decision r^2 <= r_cut^2 in FP32, redone in FP64 from the hi + lo parts when r^2 lies within
//    4e-6 r_cut^2 of the cut-off, so the pair set equals the FP64 one; local segments (avoid
//    explicit erf off) are left out here;
//  * weights from cubic tables on 1/32-wide intervals in x = alpha r (FP32, ~3e-8 absolute),
//    interval index without a conversion instruction;
//  * per-lane FP32 sums (a few pairs per lane and node), FP32 warp reduction, FP64 output sums.
constexpr int kF32Tile = 1280;
constexpr int kF32TilePad = kF32Tile + 32;  // a chunk of 32 lanes may read past the tile end (masked)
constexpr int kF32MaxDst = 128;
constexpr int kF32MaxNb = 576;    // neighbour slabs of a block: rows x slabs per row
constexpr int kF32MaxRows = 36;   // (y, z) rows of a block's neighbourhood
constexpr int kF32EvalU = 1;      // screened pairs per lane and evaluation (2: interleaved; measured slower)
constexpr int kF32Queue = 32 * kF32EvalU + 32;  // screened pairs, evaluated 32 kF32EvalU at a time
constexpr int kF32TabMax = 192;   // intervals per weight table (x = alpha r_cut <= 5.9)
constexpr float kF32Band = 4e-6f; // relative band around r_cut^2 decided in FP64
constexpr int kF32StageUnroll = 1;

struct F32Smem {
    float4 P[kF32TilePad];  // hi parts of the position, segment (int bits)
    float4 Q[kF32TilePad];  // lo parts of the position, charge x
    float2 R[kF32TilePad];  // charge y, z
    float4 tab[2][kF32TabMax];
    int32_t queue[kPairThreads / 32][kF32Queue];
    double dx[kF32MaxDst][3];
    float acc[kF32MaxDst][6];
    int32_t di[kF32MaxDst], dprev[kF32MaxDst], drow[kF32MaxDst];  // drow: the node's own row, y | z << 8
    int32_t dr_start[kMaxBlockRows], dr_cnt[kMaxBlockRows], dr_base[kMaxBlockRows + 1];
    int32_t off[kF32MaxNb + 1];
    int32_t cstart[kF32MaxNb];
    int32_t row_gA[kF32MaxRows], row_gB[kF32MaxRows];  // first cell-sorted source of the row's two runs
    int32_t row_code[kF32MaxRows];  // periodic image of the row: bits 0-1 / 2-3 = -L, 0, +L in y / z
    double dc[9];  // block constants: corner o0, o1, o2; x images sxA, sxB; cell sizes hx, h1, h2; 1 / hx
};
static_assert(sizeof(F32Smem) <= 74 * 1024, "three FP32 pair-kernel CTAs must fit in one SM's shared memory");

// U queued pairs per lane (tile indices t[u]; `valid[u]` false for the entries past the queue's end,
// which evaluate a valid entry and add nothing); the U evaluations are interleaved.
template <bool VEL, bool PSI, bool SKIP, int U>
__device__ __forceinline__ void f32_eval(const KParams& K, const F32Smem& S, float3 xh, float3 xl, float rc2,
                                         float alpha, int nf, int i, int iprev, const int (&t)[U],
                                         const bool (&valid_in)[U], float acc[6], unsigned& ninr) {
    float d0[U], d1[U], d2[U], s2[U], q0[U], q1[U], q2[U];
    bool ok[U], near[U], anynear = false;
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const float4 p = S.P[t[u]];
        const float4 q = S.Q[t[u]];
        const float2 qr = S.R[t[u]];
        d0[u] = (xh.x - p.x) + (xl.x - q.x);
        d1[u] = (xh.y - p.y) + (xl.y - q.y);
        d2[u] = (xh.z - p.z) + (xl.z - q.z);
        q0[u] = q.w;
        q1[u] = qr.x;
        q2[u] = qr.y;
        s2[u] = fmaf(d0[u], d0[u], fmaf(d1[u], d1[u], d2[u] * d2[u]));
        bool valid = valid_in[u];
        if (SKIP) {
            const int sg = __float_as_int(p.w);
            valid = valid && sg != i && sg != iprev;
        }
        ok[u] = valid && s2[u] <= rc2;
        near[u] = valid && fabsf(s2[u] - rc2) <= kF32Band * rc2;
        anynear = anynear || near[u];
    }
    if (__any_sync(0xffffffffu, anynear)) {
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (near[u]) {  // the FP64 decision on the hi + lo separation (rare)
                const float4 p = S.P[t[u]];
                const float4 q = S.Q[t[u]];
                const double e0 = ((double)xh.x + (double)xl.x) - ((double)p.x + (double)q.x);
                const double e1 = ((double)xh.y + (double)xl.y) - ((double)p.y + (double)q.y);
                const double e2 = ((double)xh.z + (double)xl.z) - ((double)p.z + (double)q.z);
                ok[u] = e0 * e0 + e1 * e1 + e2 * e2 <= K.rcut2;
            }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        ninr += __popc(__ballot_sync(0xffffffffu, ok[u]));
        const float rinv = rsqrtf(s2[u]);
        int k;
        float tt;
        f32_table_pos(s2[u] * rinv * alpha, nf, &k, &tt);
        if (VEL) {
            const float wg = f32_cubic(S.tab[1][k], tt);
            const float f = ok[u] ? wg * (rinv * rinv * rinv) : 0.0f;
            acc[0] = fmaf(f, fmaf(q1[u], d2[u], -q2[u] * d1[u]), acc[0]);
            acc[1] = fmaf(f, fmaf(q2[u], d0[u], -q0[u] * d2[u]), acc[1]);
            acc[2] = fmaf(f, fmaf(q0[u], d1[u], -q1[u] * d0[u]), acc[2]);
        }
        if (PSI) {
            const float wa = f32_cubic(S.tab[0][k], tt);
            const float f = ok[u] ? wa * rinv : 0.0f;
            acc[3] = fmaf(f, q0[u], acc[3]);
            acc[4] = fmaf(f, q1[u], acc[4]);
            acc[5] = fmaf(f, q2[u], acc[5]);
        }
    }
}

template <bool VEL, bool PSI, bool SKIP>
__global__ void __launch_bounds__(kPairThreads, 3) pair_f32_kernel(
    KParams K, CellGrid cg, int64_t Np, int64_t Ns, const int32_t* __restrict__ dst_start,
    const int32_t* __restrict__ dst_order, const double* __restrict__ nodes, const int32_t* __restrict__ idx_prev,
    const double* __restrict__ src, const int32_t* __restrict__ src_start, const int32_t* __restrict__ seg,
    double* __restrict__ vel, double* __restrict__ psi, unsigned long long* __restrict__ counters, int3 bk,
    int3 nb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    F32Smem& S = *reinterpret_cast<F32Smem*>(smem_raw);
    const int M = cg.M, G = cg.G;
    const int nc0 = cg.nc[0], nc1 = cg.nc[1], nc2 = cg.nc[2];
    const int ncc = nc0 / G;
    const int bxi = blockIdx.x % nb.x, byi = (blockIdx.x / nb.x) % nb.y, bzi = blockIdx.x / (nb.x * nb.y);
    const int cx0 = bxi * bk.x, cx1 = min(cx0 + bk.x, ncc);
    const int cy0 = byi * bk.y, cy1 = min(cy0 + bk.y, nc1);
    const int cz0 = bzi * bk.z, cz1 = min(cz0 + bk.z, nc2);
    const int ndr = (cy1 - cy0) * (cz1 - cz0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int WY = cy1 - cy0 + 2 * M, WZ = cz1 - cz0 + 2 * M, WX = (cx1 - cx0 + 2 * M) * G;
    const int nrow = WY * WZ, ncb = nrow * WX;
    const int ry0 = cy0 - M, rz0 = cz0 - M, xs0 = cx0 * G - M * G;
    // ---- prologue: destination rows, weight tables, neighbour slabs (independent loads) ----
    if (threadIdx.x < ndr) {
        const int k = threadIdx.x;
        const int yy = cy0 + k % (cy1 - cy0), zz = cz0 + k / (cy1 - cy0);
        const int64_t s0 = ((int64_t)zz * nc1 + yy) * nc0 + (int64_t)cx0 * G;
        const int a = dst_start[s0], b = dst_start[s0 + (int64_t)(cx1 - cx0) * G];
        S.dr_start[k] = a;
        S.dr_cnt[k] = b - a;
    }
    const int nf = K.ntab_c;
    for (int k = threadIdx.x; k < 2 * nf; k += kPairThreads) S.tab[k / nf][k % nf] = K.tab_c[k];
    for (int ci = threadIdx.x; ci < ncb; ci += kPairThreads) {
        const int r = ci / WX, k = ci % WX;
        int xx = xs0 + k, yy = ry0 + r % WY, zz = rz0 + r / WY;
        xx = xx < 0 ? xx + nc0 : (xx >= nc0 ? xx - nc0 : xx);
        yy = yy < 0 ? yy + nc1 : (yy >= nc1 ? yy - nc1 : yy);
        zz = zz < 0 ? zz + nc2 : (zz >= nc2 ? zz - nc2 : zz);
        const int64_t c = ((int64_t)zz * nc1 + yy) * nc0 + xx;
        const int s0 = src_start[c];
        S.cstart[ci] = s0;
        S.off[ci + 1] = src_start[c + 1] - s0;
    }
    __syncthreads();
    if (warp == 0) {  // slab counts -> concatenated offsets
        int carry = 0;
        for (int base = 0; base < ncb; base += 32) {
            const int ci = base + lane;
            int v = ci < ncb ? S.off[ci + 1] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            if (ci < ncb) S.off[ci + 1] = carry + v;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
        if (lane == 0) S.off[0] = 0;
    } else if (warp == 1) {  // destination rows -> concatenated destination offsets
        int v = lane < ndr ? S.dr_cnt[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane < ndr) S.dr_base[lane + 1] = v;
        if (lane == 0) S.dr_base[0] = 0;
    }
    // the two runs of every row in the cell-sorted arrays: slabs before / after the wrap in x
    const int kw = xs0 < 0 ? -xs0 : (xs0 + WX > nc0 ? nc0 - xs0 : WX);  // first slab past the wrap
    for (int r = threadIdx.x; r < nrow; r += kPairThreads) {
        S.row_gA[r] = S.cstart[r * WX];
        S.row_gB[r] = kw < WX ? S.cstart[r * WX + kw] : 0;
        const int yu = ry0 + r % WY, zu = rz0 + r / WY;
        S.row_code[r] = (yu < 0 ? 0 : (yu >= nc1 ? 2 : 1)) | ((zu < 0 ? 0 : (zu >= nc2 ? 2 : 1)) << 2);
    }
    if (threadIdx.x == 0) {
        const double hx = K.L[0] / nc0, h1 = K.L[1] / nc1, h2 = K.L[2] / nc2;
        S.dc[0] = cx0 * G * hx;
        S.dc[1] = cy0 * h1;
        S.dc[2] = cz0 * h2;
        S.dc[3] = xs0 < 0 ? -K.L[0] : 0.0;
        S.dc[4] = xs0 < 0 ? 0.0 : K.L[0];
        S.dc[5] = hx;
        S.dc[6] = h1;
        S.dc[7] = h2;
        S.dc[8] = nc0 / K.L[0];
    }
    __syncthreads();
    const int nd = S.dr_base[ndr];
    if (nd == 0) return;  // uniform over the CTA
    const float rc2s = (float)(K.rcut2 * (1.0 + kScreenMargin));
    const float rc2 = (float)K.rcut2;
    const float alpha = (float)K.alpha;
    const int ntot = S.off[ncb];
    const int W = 2 * M + 1;  // rows around a node's own cell in y and in z
    const int ldy = lane % W - M, ldz = lane / W - M;  // the row offset lane l examines (l < W^2)
    const double pref = K.Gamma / (4.0 * kPi);
    unsigned ninr = 0, ncand = 0;  // warp-uniform (a CTA sees far fewer than 2^32 candidates)
    for (int p0 = 0; p0 < nd; p0 += kF32MaxDst) {
        const int np = nd - p0 < kF32MaxDst ? nd - p0 : kF32MaxDst;
        // row parts per destination: at least 16 items per CTA where the block has few nodes
        const int P = np >= 16 ? 1 : (16 + np - 1) / np;
        const int nitems = np * P;
        for (int T0 = 0, T1 = 0; T0 < ntot; T0 = T1) {
            const int ra = min(last_row_le(S.off, WX, nrow, T0), nrow - 1);
            const int rf = last_row_le(S.off, WX, nrow, T0 + kF32Tile);
            T1 = S.off[rf * WX] > T0 ? S.off[rf * WX] : min(T0 + kF32Tile, ntot);
            const int rb = min(last_row_le(S.off, WX, nrow, T1 - 1) + 1, nrow);
            __syncthreads();  // previous tile consumed; previous pass written out
            if (T0 == 0) {
                for (int t = threadIdx.x; t < np; t += kPairThreads) {
                    const int tt = p0 + t;
                    int k = 0;
                    while (k + 1 < ndr && S.dr_base[k + 1] <= tt) ++k;
                    const int i = dst_order[S.dr_start[k] + tt - S.dr_base[k]];
                    S.di[t] = i;
                    const int by = cy1 - cy0;
                    S.drow[t] = ((M + k / by) << 8) | (M + k % by);  // (z, y) row coordinates, 8 bits each
                    S.dprev[t] = idx_prev[i];
#pragma unroll
                    for (int d = 0; d < 3; ++d) S.dx[t][d] = nodes[d * Np + i];
#pragma unroll
                    for (int c = 0; c < 6; ++c) S.acc[t][c] = 0.0f;
                }
            }
            // staging in units of 32 consecutive sources, kF32StageUnroll units per warp at a time
            // (their loads in flight together)
            const int nunits = (T1 - T0 + 31) >> 5;
            for (int u0 = warp; u0 < nunits; u0 += (kPairThreads / 32) * kF32StageUnroll) {
                int jj[kF32StageUnroll], tt[kF32StageUnroll], code[kF32StageUnroll];
#pragma unroll
                for (int q = 0; q < kF32StageUnroll; ++q) {
                    const int u = u0 + q * (kPairThreads / 32);
                    const int t = T0 + (u << 5) + lane;
                    tt[q] = -1;
                    jj[q] = 0;
                    code[q] = 0;
                    if (u < nunits && t < T1) {
                        int r = last_row_le(S.off, WX, nrow, T0 + (u << 5));
                        while (r + 1 < nrow && S.off[(r + 1) * WX] <= t) ++r;
                        const int rowA = S.off[r * WX], offB = S.off[r * WX + kw];
                        const bool inA = t < offB;
                        jj[q] = inA ? S.row_gA[r] + (t - rowA) : S.row_gB[r] + (t - offB);
                        tt[q] = t - T0;
                        // periodic image codes: bit 0 segment B in x; bits 1-2 / 3-4: -L, 0, +L in y / z
                        code[q] = (inA ? 0 : 1) | (S.row_code[r] << 1);
                    }
                }
                double v[kF32StageUnroll][6];
                int sgv[kF32StageUnroll];
#pragma unroll
                for (int q = 0; q < kF32StageUnroll; ++q) {
                    const int j = jj[q];
                    if (tt[q] >= 0) {
#pragma unroll
                        for (int c = 0; c < 6; ++c) v[q][c] = src[c * Ns + j];
                        sgv[q] = SKIP ? seg[j] : 0;
                    }
                }
#pragma unroll
                for (int q = 0; q < kF32StageUnroll; ++q) {
                    if (tt[q] >= 0) {
                        const int cd = code[q];
                        const double u0d = v[q][0] + S.dc[3 + (cd & 1)] - S.dc[0];
                        const double u1d = v[q][1] + (double)(((cd >> 1) & 3) - 1) * K.L[1] - S.dc[1];
                        const double u2d = v[q][2] + (double)(((cd >> 3) & 3) - 1) * K.L[2] - S.dc[2];
                        const float f0 = (float)u0d, f1 = (float)u1d, f2 = (float)u2d;
                        S.P[tt[q]] = make_float4(f0, f1, f2, __int_as_float(sgv[q]));
                        S.Q[tt[q]] = make_float4((float)(u0d - f0), (float)(u1d - f1), (float)(u2d - f2), (float)v[q][3]);
                        S.R[tt[q]] = make_float2((float)v[q][4], (float)v[q][5]);
                    }
                }
            }
            __syncthreads();
            for (int it = warp; it < nitems; it += kPairThreads / 32) {
                const int dl = it % np, part = it / np;
                const double x[3] = {S.dx[dl][0], S.dx[dl][1], S.dx[dl][2]};
                // lane l examines the row (dy, dz) = (l % W - M, l / W - M) around the node's own cell
                int a = 0, b = 0;
                if (lane < W * W) {
                    const int own = S.drow[dl];
                    const int yr = (own & 255) + ldy, zr = (own >> 8) + ldz;
                    if (yr >= 0 && yr < WY && zr >= 0 && zr < WZ) {
                        const int r = zr * WY + yr;
                        if (r >= ra && r < rb) {
                            const double h1 = S.dc[6], h2 = S.dc[7], hx = S.dc[5], inv_hx = S.dc[8];
                            const double gy = box_gap(x[1], (ry0 + yr) * h1, h1);
                            const double gz = box_gap(x[2], (rz0 + zr) * h2, h2);
                            const double gyz = gy * gy + gz * gz;
                            if (gyz <= K.rcut2) {
                                const double w = (double)sqrtf((float)(K.rcut2 - gyz)) * (1.0 + 1e-6) + 1e-9 * hx;
                                int klo = (int)floor((x[0] - w) * inv_hx) - xs0;
                                int khi = (int)floor((x[0] + w) * inv_hx) - xs0;
                                klo = klo < 0 ? 0 : klo;
                                khi = khi > WX - 1 ? WX - 1 : khi;
                                if (klo <= khi) {
                                    a = max(S.off[r * WX + klo], T0) - T0;
                                    b = min(S.off[r * WX + khi + 1], T1) - T0;
                                }
                            }
                        }
                    }
                }
                unsigned rows = __ballot_sync(0xffffffffu, a < b);
                float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                int qcount = 0;
                int32_t* Qu = S.queue[warp];
                const double xd0 = x[0] - S.dc[0], xd1 = x[1] - S.dc[1], xd2 = x[2] - S.dc[2];
                const float3 xh = make_float3((float)xd0, (float)xd1, (float)xd2);
                const float3 xl = make_float3((float)(xd0 - xh.x), (float)(xd1 - xh.y), (float)(xd2 - xh.z));
                const int i = S.di[dl], iprev = S.dprev[dl];
                for (int nrw = 0, next = part; rows; ++nrw, rows &= rows - 1) {
                    if (nrw != next) continue;  // warp-uniform: rows are dealt to the parts in turn
                    next += P;
                    const int src_lane = __ffs(rows) - 1;
                    const int ra_ = __shfl_sync(0xffffffffu, a, src_lane);
                    const int rb_ = __shfl_sync(0xffffffffu, b, src_lane);
                    ncand += rb_ - ra_;
                    for (int base = ra_; base < rb_; base += 32) {
                        const int t = base + lane;
                        const float4 p = S.P[t];
                        const float e0 = xh.x - p.x, e1 = xh.y - p.y, e2 = xh.z - p.z;
                        const bool inr = t < rb_ && fmaf(e0, e0, fmaf(e1, e1, e2 * e2)) <= rc2s;
                        const unsigned m = __ballot_sync(0xffffffffu, inr);
                        if (inr) Qu[qcount + __popc(m & ((1u << lane) - 1u))] = t;
                        qcount += __popc(m);
                        __syncwarp();
                        if (qcount >= 32 * kF32EvalU) {
                            int tq[kF32EvalU];
                            bool vq[kF32EvalU];
#pragma unroll
                            for (int u = 0; u < kF32EvalU; ++u) {
                                tq[u] = Qu[32 * u + lane];
                                vq[u] = true;
                            }
                            f32_eval<VEL, PSI, SKIP, kF32EvalU>(K, S, xh, xl, rc2, alpha, nf, i, iprev, tq, vq, acc, ninr);
                            __syncwarp();
                            if (lane < qcount - 32 * kF32EvalU) Qu[lane] = Qu[32 * kF32EvalU + lane];
                            __syncwarp();
                            qcount -= 32 * kF32EvalU;
                        }
                    }
                }
                for (int q0 = 0; q0 < qcount; q0 += 32) {  // warp-uniform remainder, one pair per lane
                    const int tq[1] = {q0 + lane < qcount ? Qu[q0 + lane] : Qu[0]};
                    const bool vq[1] = {q0 + lane < qcount};
                    f32_eval<VEL, PSI, SKIP, 1>(K, S, xh, xl, rc2, alpha, nf, i, iprev, tq, vq, acc, ninr);
                }
                __syncwarp();  // the queue is reused by the warp's next item
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    if ((c < 3 && !VEL) || (c >= 3 && !PSI)) continue;
                    float v = acc[c];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    acc[c] = v;
                }
                if (lane == 0) {
#pragma unroll
                    for (int c = 0; c < 6; ++c)
                        if ((c < 3 && VEL) || (c >= 3 && PSI)) atomicAdd(&S.acc[dl][c], acc[c]);
                }
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < np; t += kPairThreads) {
            const int64_t i = S.di[t];
            if (VEL) {
                vel[i] += pref * (double)S.acc[t][0];
                vel[Np + i] += pref * (double)S.acc[t][1];
                vel[2 * Np + i] += pref * (double)S.acc[t][2];
            }
            if (PSI) {
                psi[i] += pref * (double)S.acc[t][3];
                psi[Np + i] += pref * (double)S.acc[t][4];
                psi[2 * Np + i] += pref * (double)S.acc[t][5];
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&counters[0], (unsigned long long)ninr);
        atomicAdd(&counters[1], (unsigned long long)ncand);
    }
}

// Local term (overwrites nothing: adds into the zeroed outputs), self-interaction removal
// and, when lia_segment_fraction is set, the local integrals over the excluded sub-segments.
__global__ void __launch_bounds__(128) local_self_kernel(
    KParams K, int64_t Np, int fields, int do_local, int do_self, int do_li, double rv, double rpsi,
    const double* __restrict__ nodes, const int32_t* __restrict__ idx_prev, const double* __restrict__ d1,
    const double* __restrict__ d2, const double* __restrict__ dm, const double* __restrict__ dp,
    const double* __restrict__ points, const double* __restrict__ charges, const double* __restrict__ li_vel,
    const double* __restrict__ li_psi, double* __restrict__ vel, double* __restrict__ psi, double3 psi_bg) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Np) return;
    const bool want_v = fields & VPBS_VELOCITY, want_p = fields & VPBS_STREAMFUNCTION;
    const double pref = K.Gamma / (4.0 * kPi);
    double v[3] = {0, 0, 0}, p[3] = {0, 0, 0};
    if (do_local) {
        const double delta = sqrt(dm[i] * dp[i]);
        const double s1[3] = {d1[i], d1[Np + i], d1[2 * Np + i]};
        const double s2[3] = {d2[i], d2[Np + i], d2[2 * Np + i]};
        const double mu_inv = 1.0 / sqrt(s1[0] * s1[0] + s1[1] * s1[1] + s1[2] * s1[2]);
        if (want_v) {
            const double f = log(delta / rv) * (mu_inv * mu_inv * mu_inv);
            v[0] = pref * (f * (s1[1] * s2[2] - s1[2] * s2[1]));
            v[1] = pref * (f * (s1[2] * s2[0] - s1[0] * s2[2]));
            v[2] = pref * (f * (s1[0] * s2[1] - s1[1] * s2[0]));
        }
        if (want_p) {
            const double f = 2.0 * log(delta / rpsi) * mu_inv;
            for (int d = 0; d < 3; ++d) p[d] = pref * (f * s1[d]);
        }
    }
    if (do_self) {
        const int64_t Nq = Np * K.nquad;
        const double x[3] = {nodes[i], nodes[Np + i], nodes[2 * Np + i]};
        const int64_t ip = idx_prev[i];
        const bool explicit_erf = !K.avoid_explicit_erf && K.alpha > 0;
        double sv[3] = {0, 0, 0}, sp[3] = {0, 0, 0};
        for (int side = 0; side < 2; ++side) {
            const int64_t base = (side == 0 ? ip : i) * K.nquad;
            for (int q = 0; q < K.nquad; ++q) {
                const int64_t j = base + q;
                double r[3];
                for (int d = 0; d < 3; ++d) r[d] = deper(x[d] - points[d * Nq + j], K.L[d], K.Lh[d], K.open_domain);
                const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                const double rinv = 1.0 / rr;
                const double qc[3] = {charges[j], charges[Nq + j], charges[2 * Nq + j]};
                double fa = 1.0, fb = 0.0;
                if (explicit_erf && K.kb) {
                    // weights_longrange of the Kaiser-Bessel kernel (kaiser_bessel.jl:296-301):
                    // (F(r), r f(r)) = (1 - a, g - a) inside rcut, (1, 0) beyond
                    if (rr < K.rcut) {
                        double wa, wg;
                        ewald_weights2(K, K.alpha * rr, wa, wg);
                        fa = 1.0 - wa;
                        fb = wg - wa;
                    }
                } else if (explicit_erf) {
                    const double ar = K.alpha * rr;
                    fa = erf(ar);
                    fb = 1.1283791670955126 * ar * exp(-(ar * ar));
                }
                if (want_v) {
                    const double f = (fa - fb) * rinv * rinv * rinv;
                    sv[0] += f * (qc[1] * r[2] - qc[2] * r[1]);
                    sv[1] += f * (qc[2] * r[0] - qc[0] * r[2]);
                    sv[2] += f * (qc[0] * r[1] - qc[1] * r[0]);
                }
                if (want_p) {
                    const double f = fa * rinv;
                    for (int d = 0; d < 3; ++d) sp[d] += f * qc[d];
                }
            }
        }
        for (int d = 0; d < 3; ++d) {
            v[d] -= pref * sv[d];
            p[d] -= pref * sp[d];
        }
    }
    if (do_li) {
        for (int d = 0; d < 3; ++d) {
            v[d] += li_vel[d * Np + i];
            p[d] += li_psi[d * Np + i];
        }
    }
    if (want_v)
        for (int d = 0; d < 3; ++d) vel[d * Np + i] += v[d];
    if (want_p) {
        // streamfunction of the uniform background vorticity of unclosed filaments (zero otherwise)
        p[0] += psi_bg.x;
        p[1] += psi_bg.y;
        p[2] += psi_bg.z;
        for (int d = 0; d < 3; ++d) psi[d * Np + i] += p[d];
    }
}

}  // namespace

int build_cell_lists(vpbs_handle* h) {
    if (h->K.open_domain) return 0;
    // Cell size (internal: the pair set does not depend on it).  Where cells r_cut/2 wide would
    // hold fewer than 8 nodes, cells r_cut wide (M = 1) are used instead: the pair search is
    // then bound by per-node overhead, which grows with the (2M+1)^2 rows a node walks (1M-node
    // tangle at r_cut = L/40: 6.3 ms with M = 1 against 9.9 ms with M = 2).
    {
        const int Mu = h->P.nsubdiv;
        int M = Mu;
        if (Mu >= 2) {
            const CellGrid c2 = make_cell_grid(h->K.L, h->K.rcut, 2);
            const CellGrid c1 = make_cell_grid(h->K.L, h->K.rcut, 1);
            const double per_cell2 = (double)h->Np * c2.G / (double)c2.ncell;
            if (per_cell2 < 8.0 && c1.nc[0] >= 3 * c1.G && c1.nc[1] >= 3 && c1.nc[2] >= 3) M = 1;
        }
        if (M != h->cg.M) h->cg = make_cell_grid(h->K.L, h->K.rcut, M);
    }
    const int64_t Np = h->Np, Nq = h->Nq, ncell = h->cg.ncell;
    int rc;
    if ((rc = ensure(h, h->src_cell, sizeof(int32_t) * 2 * Nq, "src_cell"))) return rc;
    // ncell + 1 cells: the last one is the sentinel of points with non-finite coordinates
    if ((rc = ensure(h, h->src_start, sizeof(int32_t) * (ncell + 2), "src_start"))) return rc;
    if ((rc = ensure(h, h->src_fill, sizeof(int32_t) * (ncell + 1), "src_counts"))) return rc;
    if ((rc = ensure(h, h->src_sorted, sizeof(double) * 6 * Nq, "src_sorted"))) return rc;
    if ((rc = ensure(h, h->src_seg, sizeof(int32_t) * Nq, "src_seg"))) return rc;
    if ((rc = ensure(h, h->dst_cell, sizeof(int32_t) * 2 * Np, "dst_cell"))) return rc;
    if ((rc = ensure(h, h->dst_start, sizeof(int32_t) * (ncell + 2), "dst_start"))) return rc;
    if ((rc = ensure(h, h->dst_fill, sizeof(int32_t) * (ncell + 1), "dst_counts"))) return rc;
    if ((rc = ensure(h, h->dst_order, sizeof(int32_t) * Np, "dst_order"))) return rc;
    int32_t* scell = (int32_t*)h->src_cell.p;
    int32_t* srank = scell + Nq;
    int32_t* dcell = (int32_t*)h->dst_cell.p;
    int32_t* drank = dcell + Np;
    StageScope st(h, ST_CELL_LISTS);
    if ((rc = check_cuda(h, cudaMemsetAsync(h->src_fill.p, 0, sizeof(int32_t) * (ncell + 1), h->stream), "memset")))
        return rc;
    if ((rc = check_cuda(h, cudaMemsetAsync(h->dst_fill.p, 0, sizeof(int32_t) * (ncell + 1), h->stream), "memset")))
        return rc;
    cell_count_kernel<<<grid_for(Nq, 256), 256, 0, h->stream>>>(h->K, h->cg, Nq, (const double*)h->points.p, scell, srank,
                                                                (int32_t*)h->src_fill.p);
    cell_count_kernel<<<grid_for(Np, 256), 256, 0, h->stream>>>(h->K, h->cg, Np, (const double*)h->nodes.p, dcell, drank,
                                                                (int32_t*)h->dst_fill.p);
    if ((rc = exclusive_scan(h, (const int32_t*)h->src_fill.p, (int32_t*)h->src_start.p, ncell + 1, h->scan_tmp)))
        return rc;
    if ((rc = exclusive_scan(h, (const int32_t*)h->dst_fill.p, (int32_t*)h->dst_start.p, ncell + 1, h->scan_tmp)))
        return rc;
    scatter_sources_kernel<<<grid_for(Nq, 256), 256, 0, h->stream>>>(
        Nq, h->K.nquad, (const double*)h->points.p, (const double*)h->charges.p, scell, srank,
        (const int32_t*)h->src_start.p, (double*)h->src_sorted.p, (int32_t*)h->src_seg.p);
    scatter_nodes_kernel<<<grid_for(Np, 256), 256, 0, h->stream>>>(Np, dcell, drank, (const int32_t*)h->dst_start.p,
                                                                   (int32_t*)h->dst_order.p);
    h->launches += 4;  // plus the scans, counted by exclusive_scan
    return check_cuda(h, cudaGetLastError(), "cell list kernels");
}

int ewald_table_size(double xmax) { return (int)std::floor(xmax * kEwaldInvH) + 2; }

// Taylor coefficients of erfc and g(x) = erfc(x) + 2/sqrt(pi) x e^{-x^2} about the centres
// c_k = (k + 1/2)/16.  The derivatives are closed-form:
//   erfc^(n)(c) = (-1)^n 2/sqrt(pi) H_{n-1}(c) e^{-c^2}  (n >= 1, physicists' Hermite H),
//   g^(n)(c) = (1 - n) erfc^(n)(c) - c erfc^(n+1)(c)      (since g = erfc - x erfc').
// With |x - c| <= 1/32 the degree-9 remainder is below 1e-16 for all x >= 0.
void ewald_table_host(double xmax, int* ntab, double* tab) {
    const int K = ewald_table_size(xmax);
    *ntab = K;
    if (!tab) return;
    const double two_over_sqrt_pi = 2.0 / std::sqrt(kPi);
    for (int k = 0; k < K; ++k) {
        const double c = (k + 0.5) * kEwaldH;
        double H[kEwaldNC + 2];
        H[0] = 1.0;
        H[1] = 2.0 * c;
        for (int n = 1; n + 1 < kEwaldNC + 2; ++n) H[n + 1] = 2.0 * c * H[n] - 2.0 * n * H[n - 1];
        const double E = std::exp(-c * c);
        double d[kEwaldNC + 1];  // erfc^(n)(c), n = 0..NC
        d[0] = std::erfc(c);
        for (int n = 1; n <= kEwaldNC; ++n) d[n] = ((n % 2) ? -1.0 : 1.0) * two_over_sqrt_pi * H[n - 1] * E;
        double fact = 1.0;
        for (int n = 0; n < kEwaldNC; ++n) {
            if (n > 0) fact *= n;
            tab[k * kEwaldNC + n] = d[n] / fact;
            tab[(K + k) * kEwaldNC + n] = ((1.0 - n) * d[n] - c * d[n + 1]) / fact;
        }
    }
}

void table_eval_host(const double* tab, int ntab, double x, double* a, double* g) {
    int k = (int)(x * kEwaldInvH);
    k = k < ntab ? (k < 0 ? 0 : k) : ntab - 1;
    const double t = x - (k + 0.5) * kEwaldH;
    const double* ce = tab + (size_t)k * kEwaldNC;
    const double* cg = tab + (size_t)(ntab + k) * kEwaldNC;
    double va = ce[kEwaldNC - 1], vg = cg[kEwaldNC - 1];
    for (int m = kEwaldNC - 2; m >= 0; --m) {
        va = std::fma(va, t, ce[m]);
        vg = std::fma(vg, t, cg[m]);
    }
    *a = va;
    *g = vg;
}

int f32_table_size(double xmax) { return (int)std::floor(xmax * kTabCInvH) + 2; }

// Cubic interpolants of both weights on every interval [k/32, (k+1)/32], through the values of
// the FP64 table at the 4 Chebyshev points of the interval, in powers of t = 32 x - k (t in
// [0, 1]).  Over [0, xmax] they agree with the FP64 weights to ~3e-8 absolute (the FP32
// rounding of the coefficients), for the Gaussian and the Kaiser-Bessel weights alike.
void f32_table_host(const double* tab, int ntab, double xmax, float4* out) {
    const int nf = f32_table_size(xmax);
    for (int k = 0; k < nf; ++k) {
        double T[4], Va[4], Vg[4];
        for (int j = 0; j < 4; ++j) {
            T[j] = 0.5 + 0.5 * std::cos((2 * j + 1) * kPi / 8.0);
            table_eval_host(tab, ntab, (k + T[j]) / (double)kTabCInvH, &Va[j], &Vg[j]);
        }
        for (int w = 0; w < 2; ++w) {
            // solve the 4x4 Vandermonde system sum_n c_n T_j^n = V_j (Gaussian elimination, pivoting)
            double A[4][5];
            for (int j = 0; j < 4; ++j) {
                double p = 1.0;
                for (int n = 0; n < 4; ++n, p *= T[j]) A[j][n] = p;
                A[j][4] = w == 0 ? Va[j] : Vg[j];
            }
            for (int c = 0; c < 4; ++c) {
                int piv = c;
                for (int r = c + 1; r < 4; ++r)
                    if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
                for (int n = 0; n < 5; ++n) std::swap(A[c][n], A[piv][n]);
                for (int r = c + 1; r < 4; ++r) {
                    const double f = A[r][c] / A[c][c];
                    for (int n = c; n < 5; ++n) A[r][n] -= f * A[c][n];
                }
            }
            double cf[4];
            for (int c = 3; c >= 0; --c) {
                double v = A[c][4];
                for (int n = c + 1; n < 4; ++n) v -= A[c][n] * cf[n];
                cf[c] = v / A[c][c];
            }
            out[(size_t)w * nf + k] = make_float4((float)cf[0], (float)cf[1], (float)cf[2], (float)cf[3]);
        }
    }
}

void f32_table_eval_host(const float4* tabc, int nf, float x, float* a, float* g) {
    int k;
    float t;
    f32_table_pos(x, nf, &k, &t);
    *a = f32_cubic(tabc[k], t);
    *g = f32_cubic(tabc[nf + k], t);
}

int exclusive_scan(vpbs_handle* h, const int32_t* counts, int32_t* start, int64_t n, DevBuf& tmp) {
    const int64_t nblk = (n + kScanChunk - 1) / kScanChunk;
    if (nblk <= 1) {
        scan_kernel<<<1, 1024, 0, h->stream>>>(counts, start, n);
        h->launches++;
        return check_cuda(h, cudaGetLastError(), "scan kernel");
    }
    int rc;
    if ((rc = ensure(h, tmp, sizeof(int32_t) * (2 * nblk + 1), "scan partial sums"))) return rc;
    int32_t* part = (int32_t*)tmp.p;
    int32_t* part_start = part + nblk;
    scan_partials_kernel<<<(unsigned)nblk, kScanThreads, 0, h->stream>>>(counts, n, part);
    scan_kernel<<<1, 1024, 0, h->stream>>>(part, part_start, nblk);
    scan_chunks_kernel<<<(unsigned)nblk, kScanThreads, 0, h->stream>>>(counts, n, part_start, start);
    h->launches += 3;
    return check_cuda(h, cudaGetLastError(), "scan kernels");
}

template <typename T>
struct PrecTag {
    using type = T;
};

int pair_interactions(vpbs_handle* h, int fields) {
    const int64_t Np = h->Np, Nq = h->Nq;
    const bool open = h->K.open_domain;
    int rc;
    if ((rc = ensure(h, h->counters, sizeof(unsigned long long) * 2, "counters"))) return rc;
    if ((rc = check_cuda(h, cudaMemsetAsync(h->counters.p, 0, sizeof(unsigned long long) * 2, h->stream), "memset")))
        return rc;
    if (open) {
        // naive pair loop over the unsorted point data; the segment of point j is j / nquad
        if ((rc = ensure(h, h->src_sorted, sizeof(double) * 6 * Nq, "src"))) return rc;
        if ((rc = ensure(h, h->src_seg, sizeof(int32_t) * Nq, "src_seg"))) return rc;
        for (int d = 0; d < 3; ++d) {
            cudaMemcpyAsync((double*)h->src_sorted.p + d * Nq, (double*)h->points.p + d * Nq, sizeof(double) * Nq,
                            cudaMemcpyDeviceToDevice, h->stream);
            cudaMemcpyAsync((double*)h->src_sorted.p + (3 + d) * Nq, (double*)h->charges.p + d * Nq,
                            sizeof(double) * Nq, cudaMemcpyDeviceToDevice, h->stream);
        }
    }
    const int skip_local = (!h->K.avoid_explicit_erf && h->K.alpha > 0) ? 1 : 0;
    if (skip_local && open) return set_error(h, VPBS_ERR_PARAMS, "avoid_explicit_erf=false requires Ewald splitting");
    StageScope st(h, ST_PAIRS);
    const unsigned grid = grid_for(Np, 8);
    const bool v = fields & VPBS_VELOCITY, p = fields & VPBS_STREAMFUNCTION;
    const CellGrid& cg = h->cg;
    const int Wc = 2 * cg.M + 1;
    if (!open && cg.M > 0 && Wc * Wc <= kMaxRows && Wc * Wc * Wc * cg.G <= kMaxNbCells) {
        // blocks of Bc^3 cells per CTA, grown while a block holds fewer than ~24 nodes on average,
        // at least 16 CTAs per SM remain, and the neighbourhood fits the shared-memory tables and
        // stays inside one period
        const int ncc = cg.nc[0] / cg.G;
        const double ncoarse = (double)ncc * cg.nc[1] * cg.nc[2];
        const double per_cell = (double)Np / ncoarse;
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
        auto fits = [&](int nb) {
            const int w = nb + 2 * cg.M;
            return w <= ncc && w <= cg.nc[1] && w <= cg.nc[2] && w * w <= kMaxRows && w * w * w * cg.G <= kMaxNbCells &&
                   nb * nb <= kMaxBlockRows;
        };
        const bool mixed = h->P.precision == VPBS_PRECISION_MIXED;
        const int nrow_max = kF32MaxRows, ncb_max = kF32MaxNb;
        auto fits_f32 = [&](int b) {
            const int w = b + 2 * cg.M;
            return fits(b) && w * w <= nrow_max && w * w * w * cg.G <= ncb_max;
        };
        if (mixed && h->K.ewald_ntab > 0 && h->K.ntab_c > 0 && h->K.ntab_c <= kF32TabMax && fits_f32(1)) {
            // FP32 kernel: blocks grown while they hold at most ~96 nodes on average (one pass of
            // destinations) and at least 2 CTAs per SM remain; a neighbourhood of two tiles costs less
            // than a block of few nodes (1M-node tangle at r_cut = L/45: 2 x 2 x 2 cells per CTA, two
            // tiles, 2.8 ms; one cell, one tile, 4.2 ms)
            int Bc = 1;
            if (h->pair_block > 0 && fits_f32(h->pair_block)) {
                Bc = h->pair_block;  // chosen by vpbs_autotune
            } else {
                while (fits_f32(Bc + 1) && (Bc + 1) * (Bc + 1) * (Bc + 1) * per_cell <= 96.0 &&
                       ncoarse / ((double)(Bc + 1) * (Bc + 1) * (Bc + 1)) >= 2.0 * nsm)
                    ++Bc;
            }
            const int3 bk = make_int3(Bc, Bc, Bc);
            const int3 nb = make_int3((ncc + Bc - 1) / Bc, (cg.nc[1] + Bc - 1) / Bc, (cg.nc[2] + Bc - 1) / Bc);
            const size_t smem = sizeof(F32Smem);
            const unsigned nblocks = (unsigned)((int64_t)nb.x * nb.y * nb.z);
            auto launch_f32 = [&](auto kern) {
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
                kern<<<nblocks, kPairThreads, smem, h->stream>>>(
                    h->K, h->cg, Np, Nq, (const int32_t*)h->dst_start.p, (const int32_t*)h->dst_order.p,
                    (const double*)h->nodes.p, (const int32_t*)h->idx_prev.p, (const double*)h->src_sorted.p,
                    (const int32_t*)h->src_start.p, (const int32_t*)h->src_seg.p, (double*)h->vel.p, (double*)h->psi.p,
                    (unsigned long long*)h->counters.p, bk, nb);
            };
            if (skip_local) {
                if (v && p) launch_f32(pair_f32_kernel<true, true, true>);
                else if (v) launch_f32(pair_f32_kernel<true, false, true>);
                else launch_f32(pair_f32_kernel<false, true, true>);
            } else {
                if (v && p) launch_f32(pair_f32_kernel<true, true, false>);
                else if (v) launch_f32(pair_f32_kernel<true, false, false>);
                else launch_f32(pair_f32_kernel<false, true, false>);
            }
            h->launches++;
            return check_cuda(h, cudaGetLastError(), "FP32 pair kernel");
        }
        int Bc = 1;
        if (h->pair_block > 0 && fits(h->pair_block)) {
            Bc = h->pair_block;  // chosen by vpbs_autotune
        } else {
            while (Bc * Bc * Bc * per_cell < 24.0 && fits(Bc + 1) &&
                   ncoarse / ((double)(Bc + 1) * (Bc + 1) * (Bc + 1)) >= 16.0 * nsm)
                ++Bc;
        }
        const int3 bk = make_int3(Bc, Bc, Bc);
        const int3 nb = make_int3((ncc + Bc - 1) / Bc, (cg.nc[1] + Bc - 1) / Bc, (cg.nc[2] + Bc - 1) / Bc);
        const size_t smem = sizeof(TileSmem);
        const unsigned nblocks = (unsigned)((int64_t)nb.x * nb.y * nb.z);
        auto launch_tiled = [&](auto kern) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            kern<<<nblocks, kPairThreads, smem, h->stream>>>(
                h->K, h->cg, Np, Nq, (const int32_t*)h->dst_start.p, (const int32_t*)h->dst_order.p,
                (const double*)h->nodes.p, (const int32_t*)h->idx_prev.p, (const double*)h->src_sorted.p,
                (const int32_t*)h->src_start.p, (const int32_t*)h->src_seg.p, (double*)h->vel.p, (double*)h->psi.p,
                (unsigned long long*)h->counters.p, bk, nb);
        };
        auto by_fields = [&](auto skip, auto prec) {
            constexpr bool SK = decltype(skip)::value;
            using R = typename decltype(prec)::type;
            if (v && p) launch_tiled(pair_cell_kernel<true, true, SK, R>);
            else if (v) launch_tiled(pair_cell_kernel<true, false, SK, R>);
            else launch_tiled(pair_cell_kernel<false, true, SK, R>);
        };
        if (skip_local) {
            if (mixed) by_fields(std::true_type{}, PrecTag<float>{});
            else by_fields(std::true_type{}, PrecTag<double>{});
        } else {
            if (mixed) by_fields(std::false_type{}, PrecTag<float>{});
            else by_fields(std::false_type{}, PrecTag<double>{});
        }
        h->launches++;
        return check_cuda(h, cudaGetLastError(), "pair kernel");
    }
    auto launch = [&](auto kern) {
        kern<<<grid, 256, 0, h->stream>>>(h->K, h->cg, Np, Nq, (const int32_t*)h->dst_order.p, (const double*)h->nodes.p,
                                          (const int32_t*)h->idx_prev.p, (const double*)h->src_sorted.p,
                                          (const int32_t*)h->src_start.p, (const int32_t*)h->src_seg.p, (open || h->cg.M == 0) ? 0 : 1,
                                          skip_local, (double*)h->vel.p, (double*)h->psi.p,
                                          (unsigned long long*)h->counters.p);
    };
    if (h->P.precision == VPBS_PRECISION_MIXED) {
        if (v && p) launch(pair_kernel<true, true, float>);
        else if (v) launch(pair_kernel<true, false, float>);
        else launch(pair_kernel<false, true, float>);
    } else {
        if (v && p) launch(pair_kernel<true, true, double>);
        else if (v) launch(pair_kernel<true, false, double>);
        else launch(pair_kernel<false, true, double>);
    }
    h->launches++;
    return check_cuda(h, cudaGetLastError(), "pair kernel");
}

int local_and_self(vpbs_handle* h, int fields, int lia_mode, int with_pairs_self, double integration_cutoff) {
    const KParams& K = h->K;
    double rpsi, rv;
    if (integration_cutoff > 0) {
        rpsi = rv = integration_cutoff;
    } else {
        rpsi = exp(K.Delta - 1.0) * K.a / 2.0;
        rv = rpsi * exp(1.0);
    }
    const int do_local = (lia_mode == VPBS_LIA_TRUE || lia_mode == VPBS_LIA_ONLY) ? 1 : 0;
    const int do_self = with_pairs_self ? 1 : 0;
    const int do_li = (with_pairs_self && K.lia_fraction > 0) ? 1 : 0;
    // background_vorticity_correction! (BiotSavart.jl:255-286), applied with the short range: unclosed
    // filaments whose end-to-end offsets add up to p carry a mean vorticity p Gamma / V, which the
    // long range removes (k = 0 mode); the short-range streamfunction gets that of the compensating
    // uniform background, -(p Gamma / V) C
    double3 bg = make_double3(0.0, 0.0, 0.0);
    if (with_pairs_self && h->have_fil_offsets && !K.open_domain) {
        const double* p = h->offset_sum;
        double dn = 0.0, na = 0.0, nb = 0.0;
        for (int d = 0; d < 3; ++d) {
            dn += p[d] * p[d];
            na += (p[d] + K.L[d]) * (p[d] + K.L[d]);
            nb += K.L[d] * K.L[d];
        }
        // isapprox(p + Ls, Ls) (default rtol sqrt(eps)): no mean vorticity
        if (std::sqrt(dn) > std::sqrt(2.220446049250313e-16) * std::fmax(std::sqrt(na), std::sqrt(nb))) {
            const double f = -(K.Gamma / (K.L[0] * K.L[1] * K.L[2])) * h->bg_factor;
            bg = make_double3(f * p[0], f * p[1], f * p[2]);
        }
    }
    StageScope st(h, ST_LOCAL_SELF);
    local_self_kernel<<<grid_for(h->Np, 128), 128, 0, h->stream>>>(
        K, h->Np, fields, do_local, do_self, do_li, rv, rpsi, (const double*)h->nodes.p, (const int32_t*)h->idx_prev.p,
        (const double*)h->d1.p, (const double*)h->d2.p, (const double*)h->dm.p, (const double*)h->dp.p,
        (const double*)h->points.p, (const double*)h->charges.p, (const double*)h->li_vel.p,
        (const double*)h->li_psi.p, (double*)h->vel.p, (double*)h->psi.p, bg);
    h->launches++;
    return check_cuda(h, cudaGetLastError(), "local term kernel");
}

}  // namespace vpbs
