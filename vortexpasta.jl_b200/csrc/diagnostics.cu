// Diagnostics on the vorticity Fourier coefficients the long range leaves in the handle
// (src/Diagnostics/spectra.jl:84-232, spectra_helicity.jl:43-76): energy and helicity spectra
// summed over spherical shells.  Mode k (reduced grid, kx >= 0 with Hermitian symmetry) goes
// to bin n = trunc(|k| / dk + 1/2) with weight 1/2 on the kx = 0 plane and 1 elsewhere:
//   energy (vorticity state):  E_n += w |w_k|^2 / k^2 / dk          (1 / k^2 -> 1 at k = 0)
//   energy (velocity state):   E_n += w |v_k|^2 / dk,  v_k = i k x w_k / k^2 (0 at k = 0)
//   helicity:                  H_n += w 2 V Re[(i k x w_k)^* . w_k] / k^2 / dk
// where w_k are the vorticity coefficients and V the domain volume (the helicity is the same
// from either state: v_k is orthogonal to k).  One pass over the modes, per-block partial sums
// in shared memory, FP64 throughout.
//
// Coarse graining (to_coarse_grained_vorticity!, longrange.jl:160-186, 273-293): the stored
// coefficients are multiplied in place by exp(-k^2 (l^2 - l_old^2) / 2); when the reference's
// cache would hold the velocity (after a velocity evaluation), its curl i k x v_k is what gets
// filtered, i.e. the solenoidal part w_k - k (k . w_k) / k^2 of the vorticity (0 at k = 0).
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
        } else if (kind == 2) {
            // |k x w|^2 / k^4 (complex components: real and imaginary parts separately)
            const double ar0 = ky * w2.x - kz * w1.x, ai0 = ky * w2.y - kz * w1.y;
            const double ar1 = kz * w0.x - kx * w2.x, ai1 = kz * w0.y - kx * w2.y;
            const double ar2 = kx * w1.x - ky * w0.x, ai2 = kx * w1.y - ky * w0.y;
            const double k4inv = k2 == 0.0 ? 0.0 : 1.0 / (k2 * k2);
            v = k4inv * (ar0 * ar0 + ai0 * ai0 + ar1 * ar1 + ai1 * ai1 + ar2 * ar2 + ai2 * ai2);
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

__global__ void __launch_bounds__(256) coarse_grain_kernel(int nkx, int Ns1, int Ns2, double k0x, double k0y,
                                                           double k0z, double factor, int project,
                                                           double2* __restrict__ uhat, int64_t nmodes) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nmodes; u += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(u % nkx);
        const int iy = (int)((u / nkx) % Ns1);
        const int iz = (int)(u / ((int64_t)nkx * Ns1));
        const double k[3] = {k0x * ix, k0y * (iy < (Ns1 + 1) / 2 ? iy : iy - Ns1),
                             k0z * (iz < (Ns2 + 1) / 2 ? iz : iz - Ns2)};
        const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        const double op = exp(-k2 * factor);
        double2 w[3] = {uhat[u], uhat[nmodes + u], uhat[2 * nmodes + u]};
        if (project) {
            if (k2 == 0.0) {
                w[0] = w[1] = w[2] = make_double2(0.0, 0.0);
            } else {
                const double dr = (k[0] * w[0].x + k[1] * w[1].x + k[2] * w[2].x) / k2;
                const double di = (k[0] * w[0].y + k[1] * w[1].y + k[2] * w[2].y) / k2;
#pragma unroll
                for (int c = 0; c < 3; ++c) w[c] = make_double2(w[c].x - k[c] * dr, w[c].y - k[c] * di);
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) uhat[c * nmodes + u] = make_double2(op * w[c].x, op * w[c].y);
    }
}

// The held vorticity coefficients converted to the quantity the reference's cache holds:
// 1 vorticity (as stored), 2 streamfunction w / k^2, 3 velocity i k x w / k^2 (0 at k = 0).
__global__ void __launch_bounds__(256) field_of_state_kernel(int nkx, int Ns1, int Ns2, double k0x, double k0y,
                                                             double k0z, int quantity, const double2* __restrict__ uhat,
                                                             double2* __restrict__ out, int64_t nmodes) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nmodes; u += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(u % nkx);
        const int iy = (int)((u / nkx) % Ns1);
        const int iz = (int)(u / ((int64_t)nkx * Ns1));
        const double kx = k0x * ix, ky = k0y * (iy < (Ns1 + 1) / 2 ? iy : iy - Ns1),
                     kz = k0z * (iz < (Ns2 + 1) / 2 ? iz : iz - Ns2);
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double k2inv = k2 == 0.0 ? 0.0 : 1.0 / k2;
        const double2 w0 = uhat[u], w1 = uhat[nmodes + u], w2 = uhat[2 * nmodes + u];
        double2 r0 = w0, r1 = w1, r2 = w2;
        if (quantity == 2) {
            r0 = make_double2(w0.x * k2inv, w0.y * k2inv);
            r1 = make_double2(w1.x * k2inv, w1.y * k2inv);
            r2 = make_double2(w2.x * k2inv, w2.y * k2inv);
        } else if (quantity == 3) {
            r0 = make_double2(-(ky * w2.y - kz * w1.y) * k2inv, (ky * w2.x - kz * w1.x) * k2inv);
            r1 = make_double2(-(kz * w0.y - kx * w2.y) * k2inv, (kz * w0.x - kx * w2.x) * k2inv);
            r2 = make_double2(-(kx * w1.y - ky * w0.y) * k2inv, (kx * w1.x - ky * w0.x) * k2inv);
        }
        out[u] = r0;
        out[nmodes + u] = r1;
        out[2 * nmodes + u] = r2;
    }
}

}  // namespace
}  // namespace vpbs

using namespace vpbs;

extern "C" int vpbs_get_field_fourier(vpbs_handle* h, int32_t quantity, double* out, int64_t n_doubles) {
    if (!h || !out) return VPBS_ERR_ARG;
    if (quantity < 1 || quantity > 3)
        return set_error(h, VPBS_ERR_ARG, "quantity must be 1 (vorticity), 2 (streamfunction) or 3 (velocity)");
    if (!h->have_uhat)
        return set_error(h, VPBS_ERR_STATE, "no vorticity coefficients: run a long-range computation first");
    const LRSizes& S = h->lr;
    if (n_doubles != 2 * 3 * S.nmodes) return set_error(h, VPBS_ERR_ARG, "output size must be 2*3*Ns2*Ns1*(Ns0/2+1)");
    int rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (rc) return rc;
    double2* d = nullptr;
    if ((rc = check_cuda(h, cudaMalloc(&d, sizeof(double2) * 3 * S.nmodes), "cudaMalloc"))) return rc;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    const int64_t want = (S.nmodes + 255) / 256;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)nsm * 8));
    field_of_state_kernel<<<blocks, 256, 0, h->stream>>>(S.nkx, S.Ns[1], S.Ns[2], 2.0 * kPi / h->P.L[0],
                                                         2.0 * kPi / h->P.L[1], 2.0 * kPi / h->P.L[2], quantity,
                                                         (const double2*)h->uhat.p, d, S.nmodes);
    h->launches++;
    rc = check_cuda(h, cudaGetLastError(), "field kernel");
    if (!rc) rc = check_cuda(h, cudaMemcpyAsync(out, d, sizeof(double2) * 3 * S.nmodes, cudaMemcpyDeviceToHost, h->stream), "D2H");
    if (!rc) rc = check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
    cudaFree(d);
    return rc;
}

extern "C" int vpbs_coarse_grain(vpbs_handle* h, double factor, int32_t project) {
    if (!h || !std::isfinite(factor)) return VPBS_ERR_ARG;
    if (!h->have_uhat)
        return set_error(h, VPBS_ERR_STATE, "no vorticity coefficients: run a long-range computation first");
    int rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (rc) return rc;
    const LRSizes& S = h->lr;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    const int64_t want = (S.nmodes + 255) / 256;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)nsm * 8));
    coarse_grain_kernel<<<blocks, 256, 0, h->stream>>>(S.nkx, S.Ns[1], S.Ns[2], 2.0 * kPi / h->P.L[0],
                                                       2.0 * kPi / h->P.L[1], 2.0 * kPi / h->P.L[2], factor,
                                                       project ? 1 : 0, (double2*)h->uhat.p, S.nmodes);
    h->launches++;
    if ((rc = check_cuda(h, cudaGetLastError(), "coarse-graining kernel"))) return rc;
    return check_cuda(h, cudaStreamSynchronize(h->stream), "sync");
}

extern "C" int vpbs_spectrum(vpbs_handle* h, int32_t kind, double dk, double* out, int64_t nk) {
    if (!h || !out || nk < 1 || !(dk > 0)) return VPBS_ERR_ARG;
    if (kind < 0 || kind > 2)
        return set_error(h, VPBS_ERR_ARG,
                         "spectrum kind must be 0 (energy, vorticity state), 1 (helicity) or 2 (energy, velocity state)");
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
