// Diagnostics on the vorticity Fourier coefficients the long range leaves in the handle
// (src/Diagnostics/spectra.jl:84-232, spectra_helicity.jl:43-76): energy and helicity spectra
// summed over spherical shells.  Mode k (reduced grid, kx >= 0 with Hermitian symmetry) goes
// to bin n = trunc(|k| / dk + 1/2) with weight 1/2 on the kx = 0 plane and 1 elsewhere:
//   energy:   E_n += w |w_k|^2 / k^2 / dk                       (1 / k^2 -> 1 at k = 0)
//   helicity: H_n += w 2 V Re[(i k x w_k)^* . w_k] / k^2 / dk
// where w_k are the vorticity coefficients and V the domain volume.  One pass over the modes,
// per-block partial sums in shared memory, FP64 throughout.
#include <algorithm>
#include <cmath>

#include "vpbs_internal.cuh"

namespace vpbs {
namespace {

__global__ void __launch_bounds__(256) spectrum_kernel(int kind, int nkx, int Ns1, int Ns2, double k0x, double k0y,
                                                       double k0z, double dk_inv, double V, int nk,
                                                       const double2* __restrict__ uhat, int64_t nmodes,
                                                       double* __restrict__ out) {
    extern __shared__ double sbin[];
    for (int b = threadIdx.x; b < nk; b += blockDim.x) sbin[b] = 0.0;
    __syncthreads();
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nmodes; u += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(u % nkx);
        const int iy = (int)((u / nkx) % Ns1);
        const int iz = (int)(u / ((int64_t)nkx * Ns1));
        const double kx = k0x * ix;
        const double ky = k0y * (iy < (Ns1 + 1) / 2 ? iy : iy - Ns1);
        const double kz = k0z * (iz < (Ns2 + 1) / 2 ? iz : iz - Ns2);
        const double k2 = kx * kx + ky * ky + kz * kz;
        const int b = (int)(sqrt(k2) * dk_inv + 0.5);
        if (b >= nk) continue;
        const double2 w0 = uhat[u], w1 = uhat[nmodes + u], w2 = uhat[2 * nmodes + u];
        const double beta = k2 == 0.0 ? 1.0 : 1.0 / k2;
        const double factor = ix == 0 ? 0.5 : 1.0;
        double v;
        if (kind == 0) {
            v = beta * (w0.x * w0.x + w0.y * w0.y + w1.x * w1.x + w1.y * w1.y + w2.x * w2.x + w2.y * w2.y);
        } else {
            // c = k x w (complex), u_lap = i c; Re(conj(u_lap) . w) = sum_d Re(u_lap_d) Re(w_d) + Im(u_lap_d) Im(w_d)
            const double2 c0 = make_double2(ky * w2.x - kz * w1.x, ky * w2.y - kz * w1.y);
            const double2 c1 = make_double2(kz * w0.x - kx * w2.x, kz * w0.y - kx * w2.y);
            const double2 c2 = make_double2(kx * w1.x - ky * w0.x, kx * w1.y - ky * w0.y);
            const double re = (-c0.y) * w0.x + c0.x * w0.y + (-c1.y) * w1.x + c1.x * w1.y + (-c2.y) * w2.x + c2.x * w2.y;
            v = 2.0 * V * beta * re;
        }
        atomicAdd(&sbin[b], factor * v * dk_inv);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nk; b += blockDim.x)
        if (sbin[b] != 0.0) atomicAdd(&out[b], sbin[b]);
}

}  // namespace
}  // namespace vpbs

using namespace vpbs;

extern "C" int vpbs_spectrum(vpbs_handle* h, int32_t kind, double dk, double* out, int64_t nk) {
    if (!h || !out || nk < 1 || !(dk > 0)) return VPBS_ERR_ARG;
    if (kind != 0 && kind != 1) return set_error(h, VPBS_ERR_ARG, "spectrum kind must be 0 (energy) or 1 (helicity)");
    if (!h->have_uhat)
        return set_error(h, VPBS_ERR_STATE, "no vorticity coefficients: run a long-range computation first");
    if (nk > 16384) return set_error(h, VPBS_ERR_ARG, "at most 16384 spectrum bins (shared-memory partial sums)");
    int rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (rc) return rc;
    const LRSizes& S = h->lr;
    DevBuf acc;
    if ((rc = ensure(h, acc, sizeof(double) * nk, "spectrum bins"))) return rc;
    const size_t smem = sizeof(double) * nk;
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(spectrum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    rc = check_cuda(h, cudaMemsetAsync(acc.p, 0, sizeof(double) * nk, h->stream), "memset");
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    const int64_t want = (S.nmodes + 255) / 256;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)nsm * 8));
    if (!rc) {
        spectrum_kernel<<<blocks, 256, smem, h->stream>>>(
            kind, S.nkx, S.Ns[1], S.Ns[2], 2.0 * kPi / h->P.L[0], 2.0 * kPi / h->P.L[1], 2.0 * kPi / h->P.L[2],
            1.0 / dk, h->P.L[0] * h->P.L[1] * h->P.L[2], (int)nk, (const double2*)h->uhat.p, S.nmodes,
            (double*)acc.p);
        h->launches++;
        rc = check_cuda(h, cudaGetLastError(), "spectrum kernel");
    }
    if (!rc) rc = check_cuda(h, cudaMemcpyAsync(out, acc.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, h->stream), "D2H");
    if (!rc) rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
    cudaFree(acc.p);
    return rc;
}
