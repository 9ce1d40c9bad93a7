// Cheap features of a filament configuration for the parameter predictor (VPBS_NUM_FEATURES):
//   0: log10 N (nodes)
//   1: log10 (line length / L^2)  (line-length density times the period squared, cubic box)
//   2: log10 (mean segment chord / L)
//   3: log10 (min segment chord / L)
//   4..15: fractions of sampled nodes whose nearest non-local quadrature point lies at a
//          distance d with log10(d / L) in 12 bins of width 1/4 over [-3, 0) (clamped; distances
//          beyond r_cut, where the cell-list search stops, count as r_cut).
// Nodes are sampled with a stride so that at most kFeatureSample take part in the search.
#include <cmath>
#include <cstring>

#include "vpbs_internal.cuh"

namespace vpbs {
namespace {

constexpr int kFeatureSample = 32768;
constexpr int kHistBins = 12;

__device__ __forceinline__ double deper_f(double r, double L, double Lh) {
    r = (r >= Lh) ? r - L : r;
    return (r < -Lh) ? r + L : r;
}

__device__ __forceinline__ int cell_coord_f(double x, double L, int nc) {
    int c = (int)((x / L) * nc);
    return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

// Chord |x_i - x_prev(i)| of every node's incoming segment: sum (double atomics per block) and
// minimum (as ordered float bits; chords are positive).
__global__ void chord_stats_kernel(KParams K, int64_t Np, const double* __restrict__ nodes,
                                   const int32_t* __restrict__ idx_prev, double* __restrict__ sum,
                                   unsigned int* __restrict__ minbits) {
    __shared__ double ssum[8];
    __shared__ unsigned int smin[8];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double c = 0.0;
    unsigned int mb = 0x7f7fffffu;
    if (i < Np) {
        const int64_t j = idx_prev[i];  // previous node (0-based on the device)
        double s = 0;
        for (int d = 0; d < 3; ++d) {
            const double r = deper_f(nodes[d * Np + i] - nodes[d * Np + j], K.L[d], K.Lh[d]);
            s += r * r;
        }
        c = sqrt(s);
        if (c > 0) mb = __float_as_uint((float)c);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(0xffffffffu, c, o);
        mb = min(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    }
    if (lane == 0) {
        ssum[warp] = c;
        smin[warp] = mb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        unsigned int m = 0x7f7fffffu;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t += ssum[w];
            m = min(m, smin[w]);
        }
        atomicAdd(sum, t);
        atomicMin(minbits, m);
    }
}

// One warp per sampled node: nearest quadrature point of a segment j with |j - i| > 2 that is
// not one of the node's own segments, searched over the cell-list neighbourhood.
__global__ void nearest_hist_kernel(KParams K, CellGrid cg, int64_t Np, int64_t stride, const double* __restrict__ nodes,
                                    const int32_t* __restrict__ idx_prev, const double* __restrict__ src, int64_t Ns,
                                    const int32_t* __restrict__ src_start, const int32_t* __restrict__ seg,
                                    unsigned int* __restrict__ hist) {
    const int lane = threadIdx.x & 31;
    const int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t i = w * stride;
    if (i >= Np) return;
    const double x[3] = {nodes[i], nodes[Np + i], nodes[2 * Np + i]};
    const int64_t ip = idx_prev[i];
    const int M = cg.M, Mx = cg.M * cg.G;
    const int nc0 = cg.nc[0], nc1 = cg.nc[1], nc2 = cg.nc[2];
    const int cx = cell_coord_f(x[0], K.L[0], nc0), cy = cell_coord_f(x[1], K.L[1], nc1),
              cz = cell_coord_f(x[2], K.L[2], nc2);
    double best = K.rcut2;
    for (int dz = -M; dz <= M; ++dz) {
        const int zz = (cz + dz + nc2) % nc2;
        for (int dy = -M; dy <= M; ++dy) {
            const int yy = (cy + dy + nc1) % nc1;
            for (int dx = -Mx; dx <= Mx; ++dx) {
                const int xx = (cx + dx + nc0) % nc0;
                const int64_t c = ((int64_t)zz * nc1 + yy) * nc0 + xx;
                const int a = src_start[c], b = src_start[c + 1];
                for (int j = a + lane; j < b; j += 32) {
                    const int64_t sj = seg[j];
                    if ((sj - i <= 2 && i - sj <= 2) || sj == ip) continue;
                    double s = 0;
                    for (int d = 0; d < 3; ++d) {
                        const double r = deper_f(x[d] - src[d * Ns + j], K.L[d], K.Lh[d]);
                        s += r * r;
                    }
                    best = fmin(best, s);
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) {
        const double l = log10(sqrt(best) / K.L[0]);
        int bin = (int)floor((l + 3.0) * 4.0);
        bin = bin < 0 ? 0 : (bin >= kHistBins ? kHistBins - 1 : bin);
        atomicAdd(&hist[bin], 1u);
    }
}

}  // namespace
}  // namespace vpbs

using namespace vpbs;

extern "C" int vpbs_features(vpbs_handle* h, float* out, int32_t n) {
    if (!h || !out || n != VPBS_NUM_FEATURES) return VPBS_ERR_ARG;
    if (!h->have_points) return set_error(h, VPBS_ERR_STATE, "no point data: call vpbs_set_filaments or vpbs_set_points first");
    if (h->K.open_domain || h->cg.M < 1)
        return set_error(h, VPBS_ERR_STATE, "features need a periodic domain with cell lists (nsubdiv >= 1)");
    int rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (rc) return rc;
    const int64_t Np = h->Np;
    DevBuf tmp;
    if ((rc = ensure(h, tmp, 64 + sizeof(unsigned int) * (kHistBins + 1), "feature scratch"))) return rc;
    double* dsum = (double*)tmp.p;
    unsigned int* minbits = (unsigned int*)((char*)tmp.p + 8);
    unsigned int* hist = (unsigned int*)((char*)tmp.p + 64);
    const unsigned int init_min = 0x7f7fffffu;
    cudaMemsetAsync(tmp.p, 0, 64 + sizeof(unsigned int) * (kHistBins + 1), h->stream);
    cudaMemcpyAsync(minbits, &init_min, sizeof(init_min), cudaMemcpyHostToDevice, h->stream);
    chord_stats_kernel<<<grid_for(Np, 256), 256, 0, h->stream>>>(h->K, Np, (const double*)h->nodes.p,
                                                                (const int32_t*)h->idx_prev.p, dsum, minbits);
    const int64_t stride = (Np + kFeatureSample - 1) / kFeatureSample;
    const int64_t nsample = (Np + stride - 1) / stride;
    nearest_hist_kernel<<<grid_for(nsample, 8), 256, 0, h->stream>>>(
        h->K, h->cg, Np, stride, (const double*)h->nodes.p, (const int32_t*)h->idx_prev.p,
        (const double*)h->src_sorted.p, h->Nq, (const int32_t*)h->src_start.p, (const int32_t*)h->src_seg.p, hist);
    h->launches += 2;
    double hsum = 0;
    unsigned int hmin = 0, hh[kHistBins];
    rc = check_cuda(h, cudaGetLastError(), "feature kernels");
    if (!rc) rc = check_cuda(h, cudaMemcpyAsync(&hsum, dsum, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "copy");
    if (!rc) rc = check_cuda(h, cudaMemcpyAsync(&hmin, minbits, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream), "copy");
    if (!rc) rc = check_cuda(h, cudaMemcpyAsync(hh, hist, sizeof(hh), cudaMemcpyDeviceToHost, h->stream), "copy");
    if (!rc) rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
    cudaFree(tmp.p);
    if (rc) return rc;
    const double L = h->K.L[0];
    float minc;
    std::memcpy(&minc, &hmin, sizeof(float));
    out[0] = (float)std::log10((double)Np);
    out[1] = (float)std::log10(hsum / (L * L));
    out[2] = (float)std::log10(hsum / Np / L);
    out[3] = (float)std::log10((double)minc / L);
    for (int b = 0; b < kHistBins; ++b) out[4 + b] = (float)((double)hh[b] / (double)nsample);
    return 0;
}
