/*
 * vp_oracle.h -- CPU FP64 restatement of VortexPasta's Ewald-split Biot-Savart
 * evaluation on filament nodes.  TEST INFRASTRUCTURE ONLY: this library is the
 * checker the CUDA path is compared against (tests, smoke(), and the CPU
 * baseline leg of bench.py).  It is never linked into, called by, or shipped
 * with the product library.
 *
 * Parity status: the reference (Julia) cannot be executed in this environment,
 * so the oracle is pinned against the reference's own known-answer tests
 * (analytic vortex-ring velocity/streamfunction, exact Fourier sums for the
 * long-range part, exact pair counts, independence from the Ewald splitting
 * parameter) rather than against reference outputs.
 *
 * All reference citations are relative to the VortexPasta.jl source tree.
 */
#ifndef VP_ORACLE_H
#define VP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double Gamma, a, Delta;          /* circulation, core size, core parameter */
    double L[3];                     /* periods; <= 0 means open (infinite) */
    double alpha;                    /* Ewald splitting parameter; 0 => NoSplitting */
    double rcut;                     /* short-range cut-off (ignored if alpha == 0) */
    int    Ns[3];                    /* Fourier modes per dimension (long range) */
    double sigma;                    /* NUFFT oversampling factor */
    int    m;                        /* NUFFT kernel half-support (grid points) */
    int    nquad;                    /* Gauss-Legendre points per segment */
    int    nquad_near;               /* GL points for lia_segment_fraction integrals */
    double lia_segment_fraction;     /* <= 0 means `nothing` (full segments) */
    int    avoid_explicit_erf;       /* 1 (reference default) or 0 */
    int    truncate_spherical;       /* longrange_truncate_spherical */
    int    nsubdiv;                  /* cell-list subdivisions M; 0 => naive pair loop */
    int    longrange_exact;          /* 1 => ExactSumBackend instead of NUFFT */
    int    nthreads;                 /* OpenMP threads (<= 0: default) */
    int    splitting;                /* 0: Gaussian (alpha) / none; 1: Kaiser-Bessel */
    double kb_beta;                  /* Kaiser-Bessel shape parameter */
    double kb_rtol;                  /* Kaiser-Bessel rtol (Chebyshev truncation) */
    const double* fil_offsets;       /* [nfil][3] end-to-end offsets of the filaments (NULL: all
                                        zero, closed filaments; closed_filament.jl:118-132) */
    int    nufft_kernel;             /* 0: ES kernel; 1: backward Kaiser-Bessel kernel */
} vpo_params;

/* Kaiser-Bessel short-range weights 1 - F(r) and 1 - F(r) + r f(r) from the truncated
 * Chebyshev series (reference: src/BiotSavart/splitting/kaiser_bessel.jl:139-147, 282-292;
 * splitting/chebyshev.jl:33-172).  Returns the number of even coefficients kept in f, or -1. */
int vpo_kb_weights(double beta, double rcut, double rtol, const double* r, long n, double* a, double* g);

typedef struct {
    int64_t pairs_in_range;          /* pairs with r^2 <= rcut^2 (short range) */
    int64_t pairs_candidates;        /* pairs examined */
    int     fft_n[3];                /* oversampled FFT grid size */
    double  es_beta;                 /* ES kernel shape parameter */
} vpo_stats;

/* Gauss-Legendre rule on [0, 1] (reference: src/Quadratures/Quadratures.jl:52-56, 147-169). */
void vpo_gl_rule(int n, double* zeta, double* w);

/* Oversampled FFT size used by the NUFFT: smallest even 2^a 3^b 5^c >= sigma*Ns. */
int vpo_fft_size(int Ns, double sigma);

/* Point data of add_point_charges! (reference: src/BiotSavart/pointdata_impl.jl:41-108).
 * nodes_xyz: AoS [Np][3]; offsets[nfil+1] (filament f owns nodes offsets[f]..offsets[f+1]-1).
 * Outputs (AoS [.][3] unless scalar): nodes (folded), idx_prev (0-based), d1, d2 (s', s'' at
 * nodes), dm, dp (subsegment lengths), points, charges ([Np*nquad][3]). */
int vpo_point_data(const vpo_params* p, int nfil, const int64_t* offsets, const double* nodes_xyz,
                   double* nodes_f, int32_t* idx_prev, double* d1, double* d2,
                   double* dm, double* dp, double* points, double* charges);

/* Vorticity Fourier coefficients (after the Gamma/V prefactor and Hermitian-symmetry
 * zeroing), on the reduced grid [Ns0/2+1][Ns1][Ns2] x-fastest, 3 components, complex
 * interleaved: out[((c*Ns2 + iz)*Ns1 + iy)*(Ns0/2+1) + ix] (re, im). */
int vpo_vorticity_fourier(const vpo_params* p, int64_t Nq, const double* points, const double* charges,
                          double* uhat_out, vpo_stats* st);

/* Streamfunction factor of a uniform background vorticity: 1 / (4 alpha^2) (Gaussian) or
 * int_0^rcut r^2 f(r) dr / 2 (Kaiser-Bessel); reference: BiotSavart.jl:255-286. */
double vpo_background_factor(const vpo_params* p);

/* Full compute_on_nodes! (reference: src/BiotSavart/BiotSavart.jl:395-612).
 * lia_mode: 0 = Val(false), 1 = Val(true), 2 = Val(:only).
 * vel_out / psi_out: AoS [Np][3] or NULL when that field is not requested. */
int vpo_compute_on_nodes(const vpo_params* p, int nfil, const int64_t* offsets, const double* nodes_xyz,
                         int lia_mode, int shortrange, int longrange,
                         double* vel_out, double* psi_out, vpo_stats* st);

#ifdef __cplusplus
}
#endif
#endif
