/*
 * vpbs.h -- C ABI of libvpbs.so, a CUDA (sm_100a) implementation of VortexPasta's
 * Ewald-split Biot-Savart velocity / streamfunction evaluation on filament nodes.
 *
 * The library is a drop-in for the CellListsBackend + NonuniformFFTsBackend pair of
 * VortexPasta.BiotSavart.  Every entry point below names the reference interface it
 * replaces (paths relative to the VortexPasta.jl source tree).  All functions
 * return 0 on success and a negative vpbs_status on failure; the message is then
 * available from vpbs_last_error(handle) (or vpbs_last_error(NULL) for failures of
 * vpbs_create).
 *
 * Ownership: the caller owns every host array it passes; the library owns all device
 * memory, cuFFT plans, streams and pinned staging buffers of a handle, and retains no
 * caller pointer after a call returns.  Calls on one handle must be serialised by the
 * caller; distinct handles may be used concurrently from different threads (each has
 * its own CUDA stream unless vpbs_set_stream is used).
 */
#ifndef VPBS_H
#define VPBS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vpbs_handle vpbs_handle;

typedef enum {
    VPBS_OK = 0,
    VPBS_ERR_ARG = -1,        /* invalid argument (null pointer, bad size, bad flag) */
    VPBS_ERR_PARAMS = -2,     /* inconsistent parameters (e.g. r_cut too large) */
    VPBS_ERR_OOM = -3,        /* device or pinned-host allocation failed */
    VPBS_ERR_CUDA = -4,       /* CUDA runtime or cuFFT error */
    VPBS_ERR_STATE = -5,      /* call out of order (e.g. compute before set_points) */
    VPBS_ERR_TIMEOUT = -6     /* a bounded device-side wait gave up */
} vpbs_status;

/* Output field selection bits for vpbs_compute and friends. */
#define VPBS_VELOCITY 1
#define VPBS_STREAMFUNCTION 2

/* LIA modes of compute_on_nodes! (src/BiotSavart/BiotSavart.jl:395-404). */
#define VPBS_LIA_FALSE 0
#define VPBS_LIA_TRUE 1
#define VPBS_LIA_ONLY 2

/* Arithmetic forms. */
#define VPBS_PRECISION_FP64 0 /* plain method: everything in double precision */
#define VPBS_PRECISION_MIXED 1 /* FP32 bulk (pairs, spreading, FFT, interpolation); FP64
                                  positions, separations, local term, final accumulation */

/* NUFFT spreading kernels.  The reference passes no kernel to NonuniformFFTs.jl (compat "0.8.2, 0.9",
 * not in its tree), whose default is a Kaiser-Bessel-type kernel; its exact shape parameter, evaluation
 * and FFT-size rounding cannot be pinned here, so results agree with the reference's to the NUFFT
 * tolerance (~1e-6 at m = 4), not bit for bit. */
#define VPBS_NUFFT_ES 0              /* exponential of semicircle, beta = 0.97 pi m (2 - 1/sigma) */
#define VPBS_NUFFT_KAISER_BESSEL 1   /* backward Kaiser-Bessel, beta = 0.995 pi m (2 - 1/sigma) */

/* Ewald splitting kernels (src/BiotSavart/splitting/splitting.jl:1-47). */
#define VPBS_SPLITTING_GAUSSIAN 0      /* GaussianSplitting, or NoSplitting when alpha == 0 */
#define VPBS_SPLITTING_KAISER_BESSEL 1 /* KaiserBesselSplitting (splitting/kaiser_bessel.jl) */

/* Parameters: the union of ParamsCommon, ParamsShortRange and ParamsLongRange
 * (src/BiotSavart/params.jl:8-30, 74-115, 141-152) plus the two backends
 * (CellListsBackend, shortrange/backends/cell_lists.jl:64-87; NonuniformFFTsBackend,
 * longrange/backends/nonuniformffts.jl:97-126).  GaussianSplitting is described by
 * (alpha, rcut, Ns) already derived by the caller (splitting/gaussian.jl:133-200);
 * alpha == 0 selects NoSplitting (open domain, naive pair sum, no long range).
 * KaiserBesselSplitting is described by (kb_beta, rcut, Ns, kb_rtol) already derived by the
 * caller (kaiser_bessel.jl:165-223); alpha is ignored for it.  kb_rtol sets the truncation
 * of the Chebyshev series of the kernel and of its integral (kaiser_bessel.jl:139-147), as
 * in the reference. */
typedef struct {
    double Gamma;                 /* circulation */
    double a;                     /* vortex core size */
    double Delta;                 /* core vorticity-profile coefficient */
    double L[3];                  /* periods (ignored when alpha == 0) */
    double alpha;                 /* Ewald splitting parameter, 0 => NoSplitting */
    double rcut;                  /* short-range cut-off distance */
    int32_t Ns[3];                /* Fourier modes per direction */
    double sigma;                 /* NUFFT oversampling factor (reference default 1.5) */
    int32_t m;                    /* NUFFT kernel half-support (HalfSupport(m)) */
    int32_t nquad;                /* quadrature points per segment (1..16) */
    double quad_zeta[16];         /* quadrature nodes on [0, 1] */
    double quad_w[16];            /* quadrature weights on [0, 1] */
    int32_t nquad_near;           /* quadrature_near_singularity (1..16) */
    double quad_near_zeta[16];
    double quad_near_w[16];
    double lia_segment_fraction;  /* in (0, 1]; <= 0 means `nothing` */
    int32_t avoid_explicit_erf;   /* reference default 1 */
    int32_t truncate_spherical;   /* longrange_truncate_spherical */
    int32_t nsubdiv;              /* CellListsBackend subdivisions M (reference default 2) */
    int32_t precision;            /* VPBS_PRECISION_* */
    int32_t device;               /* CUDA device ordinal */
    int32_t splitting;            /* VPBS_SPLITTING_* (0, the zero-initialised value: Gaussian) */
    double kb_beta;               /* Kaiser-Bessel shape parameter beta */
    double kb_rtol;               /* Kaiser-Bessel relative accuracy rtol */
    int32_t nufft_kernel;         /* VPBS_NUFFT_* (0, the zero-initialised value: ES) */
} vpbs_params;

/* Structure-of-arrays view of a vector of Vec3 (the layout of a StructVector{Vec3}). */
typedef struct { const double* x; const double* y; const double* z; } vpbs_cvec3;
typedef struct { double* x; double* y; double* z; } vpbs_vec3;

/* BiotSavart.init_cache(params) -> BiotSavartCache  (src/BiotSavart/cache.jl:40-49;
 * init_cache_short, shortrange/backends/cell_lists.jl:103-115; init_cache_long_ewald,
 * longrange/backends/nonuniformffts.jl:153-171).  Validates the parameters with the
 * reference's rules (params.jl:99-106; CellLists.jl:135-147). */
int vpbs_create(const vpbs_params* params, vpbs_handle** out);

/* Releases every resource of the handle. */
int vpbs_destroy(vpbs_handle* h);

/* Message of the last failure on `h` (or of the last failed vpbs_create when h is NULL). */
const char* vpbs_last_error(const vpbs_handle* h);

/* Run all work of `h` on the caller's CUDA stream (a cudaStream_t; NULL restores the
 * handle's own stream).  Replaces the device selection of activate_device!
 * (src/BiotSavart/ka_utils.jl:38-49). */
int vpbs_set_stream(vpbs_handle* h, void* stream);

/* add_point_charges!(pointdata, fs, params) on the device (src/BiotSavart/pointdata_impl.jl:41-108):
 * from closed-filament nodes (AoS [Np][3], filament f owns nodes offsets[f]..offsets[f+1]-1)
 * builds chordal knots, periodic quintic splines (src/Filaments/spline/quintic.jl:9-100) and
 * the point data (folded nodes, previous-node indices, s' and s'' on nodes, sub-segment
 * lengths, quadrature points and charges).  `offsets` is always a host array; `nodes_xyz` is a
 * host pointer (copied through pinned staging) when `on_device` = 0, or a device pointer read
 * in place on the handle's stream when `on_device` = 1. */
int vpbs_set_filaments(vpbs_handle* h, int64_t nfil, const int64_t* offsets, const double* nodes_xyz,
                       int32_t on_device);

/* End-to-end offsets of unclosed (infinite) filaments, ClosedFilament's Xoffset
 * (src/Filaments/closed_filament.jl:118-132, 196-207): host [nfil][3], or NULL / all zero for closed
 * filaments.  They apply to the following vpbs_set_filaments / vpbs_set_filament_list /
 * vpbs_set_staged_filaments calls (which must pass nfil filaments) and RK4 steps, until changed.
 * The splines then interpolate the periodic y_i = X_i - (t_i / T) offset (spline.jl:163-194,
 * quintic.jl:9-17), and when the offsets add up to p != 0 the short range adds the streamfunction
 * of the compensating background vorticity, -(p Gamma / V) C, to every node
 * (background_vorticity_correction!, src/BiotSavart/BiotSavart.jl:255-286; C = 1 / (4 alpha^2),
 * or int_0^rcut r^2 f(r) dr / 2 for the Kaiser-Bessel splitting). */
int vpbs_set_filament_offsets(vpbs_handle* h, int64_t nfil, const double* offsets_xyz);

/* Plugin-contract entry: PointData computed by the caller (the reference computes it on the
 * host in add_point_charges!).  Layout per src/BiotSavart/pointdata.jl:21-31: nodes, derivatives
 * and charges as SoA views; node_idx_prev is 1-based as in the reference; points/charges hold
 * nquad entries per node, point index nquad*(n-1)+q on segment [n, n+1]. Host pointers. */
int vpbs_set_points(vpbs_handle* h, int64_t Np, vpbs_cvec3 nodes, const int32_t* node_idx_prev,
                    vpbs_cvec3 deriv1, vpbs_cvec3 deriv2, const double* delta_minus,
                    const double* delta_plus, vpbs_cvec3 points, vpbs_cvec3 charges);

/* compute_on_nodes!(fields, cache, fs; LIA, shortrange, longrange) without the host
 * transfers (src/BiotSavart/BiotSavart.jl:515-612): results stay in device memory.
 * fields: VPBS_VELOCITY | VPBS_STREAMFUNCTION.  integration_cutoff <= 0 means `nothing`
 * (local_integrals.jl:115-126).  Asynchronous on the handle's stream. */
int vpbs_compute(vpbs_handle* h, int32_t fields, int32_t lia_mode, int32_t shortrange, int32_t longrange,
                 double integration_cutoff);

/* The reference's default device split (src/BiotSavart/BiotSavart.jl:535-605; the short range on
 * device 2, shortrange/backends/cell_lists.jl:7,50,81; the long range on device 1,
 * longrange/backends/nonuniformffts.jl:108-118): two handles evaluate the two parts of the same
 * filaments concurrently (vpbs_compute with shortrange = 1, longrange = 0 on one and the reverse on the
 * other), and this call adds the computed `fields` of `src` into those of `dst`, on dst's stream after
 * src's work.  When src lives on another GPU its field crosses once, by a peer copy into dst's memory.
 * Both handles must hold the same nodes.  Asynchronous. */
int vpbs_add_field(vpbs_handle* dst, vpbs_handle* src, int32_t fields);

/* copy_output_values_on_nodes! (src/BiotSavart/BiotSavart.jl:628-715): device -> host copy of a
 * computed field (VPBS_VELOCITY or VPBS_STREAMFUNCTION) in node order, AoS [Np][3].
 * accumulate = 1 adds to the existing host values (op = +), 0 overwrites.  Synchronises the
 * handle's stream. */
int vpbs_get(vpbs_handle* h, int32_t field, double* out_xyz, int32_t accumulate);

/* Per-filament variants for hosts that keep one array per filament (the reference's
 * Vector of filaments): vpbs_set_filament_list takes nfil host pointers to AoS [counts[f]][3]
 * node arrays (same semantics as vpbs_set_filaments with on_device = 0); vpbs_get_filament_list
 * writes a computed field into nfil host AoS arrays laid out like the filaments of the last
 * vpbs_set_filaments / vpbs_set_filament_list.  Both copy through pinned staging with up to 8
 * host threads. */
int vpbs_set_filament_list(vpbs_handle* h, int64_t nfil, const double* const* nodes, const int64_t* counts);
int vpbs_get_filament_list(vpbs_handle* h, int32_t field, double* const* out, int64_t nfil);

/* Staging without an intermediate copy, for hosts that assemble the inputs themselves:
 * vpbs_stage_filaments returns pinned host buffers for nfil+1 offsets and 3 Np AoS node
 * coordinates (valid until the next staging call on h) that the caller fills; then
 * vpbs_set_staged_filaments(h, nfil) proceeds as vpbs_set_filaments with host nodes.
 * vpbs_get_staged returns a pinned AoS [Np][3] copy of a computed field (node order), valid until
 * the next call on h.  Both synchronise the handle's stream as needed. */
int vpbs_stage_filaments(vpbs_handle* h, int64_t nfil, int64_t Np, int64_t** offsets, double** nodes);
int vpbs_set_staged_filaments(vpbs_handle* h, int64_t nfil);
int vpbs_get_staged(vpbs_handle* h, int32_t field, const double** aos);

/* Same as vpbs_get but into SoA host arrays. */
int vpbs_get_soa(vpbs_handle* h, int32_t field, vpbs_vec3 out, int32_t accumulate);

/* Device pointers of a computed field (SoA, Np doubles each), valid until the next call that
 * changes the number of nodes or vpbs_destroy. */
int vpbs_device_field(vpbs_handle* h, int32_t field, double** x, double** y, double** z);

/* get_longrange_field_fourier (src/BiotSavart/cache.jl:72-83): the vorticity Fourier
 * coefficients of the last long-range computation (state :vorticity, unsmoothed), as
 * complex-interleaved doubles [3][Ns2][Ns1][Ns0/2+1] (x fastest).  `n_doubles` must equal
 * 2*3*Ns2*Ns1*(Ns0/2+1).  Synchronises the handle's stream. */
int vpbs_get_uhat(vpbs_handle* h, double* out, int64_t n_doubles);

/* Read back the device point data (the fields of PointData, src/BiotSavart/pointdata.jl:21-31,
 * as exposed by cache.pointdata): which = 0 nodes (folded, SoA 3*Np), 1 s' on nodes (3*Np),
 * 2 s'' on nodes (3*Np), 3 delta_minus (Np), 4 delta_plus (Np), 5 points (SoA 3*Nq),
 * 6 charges (SoA 3*Nq), 7 node_idx_prev (Np int32, 0-based).  `n_elems` must match.
 * Synchronises the handle's stream. */
int vpbs_get_pointdata(vpbs_handle* h, int32_t which, void* out, int64_t n_elems);

/* Short-range counters of the last computation: in-range pairs (r^2 <= r_cut^2) and
 * examined candidate pairs.  Synchronises the handle's stream. */
int vpbs_pair_counts(vpbs_handle* h, int64_t* in_range, int64_t* candidates);

/* Oversampled FFT grid size chosen for Ns modes at oversampling sigma (smallest even
 * 2^a 3^b 5^c >= sigma*Ns); the reference delegates this to NonuniformFFTs.jl. */
int32_t vpbs_fft_size(int32_t Ns, double sigma);

/* Number of the library's own kernels launched on `h` since creation (cuFFT's kernels are not
 * counted).  Measurement support; no counterpart in the reference. */
int64_t vpbs_launch_count(const vpbs_handle* h);

/* Per-stage CUDA-event timing on the handle's stream, the device-side analogue of the
 * reference's TimerOutputs sections (src/BiotSavart/BiotSavart.jl:417-509).  Enable with
 * vpbs_stage_timing(h, 1); vpbs_stage_times fills ms[0..VPBS_NUM_STAGES) with the time of each
 * stage since the previous query (synchronises the stream); vpbs_stage_name(i) names stage i. */
#define VPBS_NUM_STAGES 9
int vpbs_stage_timing(vpbs_handle* h, int32_t enable);
int vpbs_stage_times(vpbs_handle* h, double* ms, int32_t n);
const char* vpbs_stage_name(int32_t i);

/* Allocation-free variant of the point-data computation of vpbs_set_filaments, with no
 * counterpart in the reference.  It is for callers that cannot allocate device memory: code
 * running where cudaMalloc is forbidden or unsafe (under an external memory pool that owns all
 * device memory, inside another runtime's stream-ordered region, or in a binding that can only
 * hand over buffers it already owns).  It calls no cudaMalloc, cudaFree or allocating library
 * routine: the spline solve's intermediates (knots, B-spline coefficients, banded factors) live
 * in one file-scope device array of about 6 MB that every GPU loading the library holds until
 * the process exits.
 *
 * Inputs: params (quadrature rule, periods, lia_segment_fraction, device), `nfil` filaments with
 * host `offsets[nfil+1]`, device AoS nodes `nodes_xyz` [Np][3]; `stream` (cudaStream_t, may be
 * NULL).  Outputs (device pointers, same layouts as vpbs_get_pointdata): nodes, s', s'' (SoA
 * 3*Np), node_idx_prev (Np, 0-based), delta_minus, delta_plus (Np), points, charges (SoA 3*Nq).
 * Limits: at most VPBS_NOALLOC_MAX_NODES nodes and VPBS_NOALLOC_MAX_FILAMENTS filaments; larger
 * inputs are rejected with VPBS_ERR_ARG.  `nodes_xyz` and every output must be device (or managed)
 * memory of params->device, else VPBS_ERR_ARG; the caller's current device is restored on return.
 * Every call looks up the array's device address (cudaGetSymbolAddress, no allocation).  Under
 * CUDA's lazy module loading (the default since CUDA 12.2) the driver materialises the array, and
 * this file's kernels, at the first call on each device: make one warm-up call on every device
 * before an external pool claims the device memory, and before any stream capture.
 * All calls share the one array: calls that overlap on the GPU (other streams, other threads)
 * race and must be serialised by the caller.  Errors: vpbs_last_error(NULL). Asynchronous. */
#define VPBS_NOALLOC_MAX_NODES 32768
#define VPBS_NOALLOC_MAX_FILAMENTS 4096
int vpbs_point_data_noalloc(const vpbs_params* params, int64_t nfil, const int64_t* offsets, const double* nodes_xyz,
                            void* stream, double* nodes, int32_t* node_idx_prev, double* deriv1, double* deriv2,
                            double* delta_minus, double* delta_plus, double* points, double* charges);

/* Host evaluation of the pair kernel's Ewald weight tables (same coefficients and Horner/FMA
 * order as on the device): erfc(x) and erfc(x) + 2/sqrt(pi) x exp(-x^2) for x in [0, xmax]
 * (xmax = alpha * rcut).  The device replaces the reference's erfc/exp calls
 * (splitting/gaussian.jl:273-279) by these degree-9 Taylor tables; this entry exists to test
 * them.  No counterpart in the reference. */
int vpbs_ewald_table_eval(double xmax, const double* x, int64_t n, double* erfc_out, double* g_out);

/* Host evaluation of the Kaiser-Bessel short-range weights a = 1 - F(r) and g = 1 - F(r) + r f(r)
 * for r in [0, rcut]: from the pair kernel's tables (a_table, g_table) and from the truncated
 * Chebyshev series they are fitted to (a_series, g_series), built with the reference's rules
 * (splitting/kaiser_bessel.jl:139-147, splitting/chebyshev.jl:73-172).  Any output may be NULL.
 * Exists to test the tables and the series; no counterpart in the reference. */
int vpbs_kb_weights(double beta, double rcut, double rtol, const double* r, int64_t n, double* a_table,
                    double* g_table, double* a_series, double* g_series);

/* Host evaluation of the mixed form's FP32 pair-kernel weights (the cubic tables on 1/32-wide
 * intervals, built as on the device and evaluated with the same float operations): a = erfc(alpha r)
 * and g = erfc(alpha r) + 2/sqrt(pi) alpha r exp(-(alpha r)^2) for splitting = VPBS_SPLITTING_GAUSSIAN
 * (splitting/gaussian.jl:273-279), a = 1 - F(r) and g = 1 - F(r) + r f(r) of the truncated Chebyshev
 * series for VPBS_SPLITTING_KAISER_BESSEL (kaiser_bessel.jl:139-147; alpha ignored), for r in
 * [0, rcut].  Exists to test the tables; no counterpart in the reference. */
int vpbs_f32_weights_eval(int32_t splitting, double alpha, double rcut, double kb_beta, double kb_rtol, const double* r,
                          int64_t n, float* a, float* g);

/* Host evaluation of the device's periodic helpers (the same inline code, periodic.cuh): x folded
 * into [0, L) (min_distance.jl:5-20; O(1) for any x, NaN for a non-finite x) and the cell index
 * trunc(folded / L * nc) clamped to [0, nc) (CellLists.jl:194-204, 0-based), or the sentinel nc for
 * a non-finite coordinate.  Either output may be NULL.  Exists to test them; no counterpart in the
 * reference. */
int vpbs_periodic_eval(double L, int32_t nc, const double* x, int64_t n, double* folded, int64_t* cell);

/* Host copies dst[k] <- src[k] of bytes[k] each (k < n) on the library's copy threads, the routine the
 * host-buffer entry points stage their inputs and outputs with: blocks split into pieces of about
 * 1 MB, small blocks grouped, a pool of up to 7 threads plus the caller (created on first use, and
 * again in a forked child).  Host memory only; no GPU needed.  Exists to test the staging; no
 * counterpart in the reference. */
int vpbs_host_copies(int64_t n, void* const* dst, const void* const* src, const size_t* bytes);

/* Measured CUDA-core FMA throughput of `device` in TFLOP/s (fp64 = 1: double, 0: float); the
 * denominator of the pair kernel's roofline.  Measurement support; no counterpart in the
 * reference. */
int vpbs_fma_throughput(int32_t device, int32_t fp64, double* tflops);

/* ---- Diagnostics (src/Diagnostics/spectra.jl:84-232, spectra_helicity.jl:43-76) ---- */

/* Energy or helicity spectrum of the vorticity coefficients w_k held by the handle (the field of
 * vpbs_get_uhat), summed over spherical shells of width dk: out[n] for k_n = n dk,
 * n = 0..nk-1 (bin n = trunc(|k|/dk + 1/2), weight 1/2 on the kx = 0 plane).  kind 0: energy as
 * the reference computes it from a vorticity-state cache, sum of |w_k|^2/k^2/dk; kind 2: energy
 * as from a velocity-state cache (the state after a velocity evaluation), sum of |v_k|^2/dk with
 * v_k = i k x w_k / k^2; kind 1: helicity, sum of 2 V Re[(i k x w_k)^* . w_k]/k^2/dk (the same
 * from either state).  Synchronous; host output. */
int vpbs_spectrum(vpbs_handle* h, int32_t kind, double dk, double* out, int64_t nk);

/* get_longrange_field_fourier for a given cache state: the held coefficients as quantity
 * 1 = vorticity (as vpbs_get_uhat), 2 = streamfunction w_k / k^2 (after
 * compute_streamfunction_fourier!, longrange.jl:102-125), 3 = velocity i k x w_k / k^2 (after
 * compute_velocity_fourier!, longrange.jl:128-156); 0 at k = 0 for 2 and 3.  Layout and size as
 * vpbs_get_uhat.  Synchronous. */
int vpbs_get_field_fourier(vpbs_handle* h, int32_t quantity, double* out, int64_t n_doubles);

/* to_coarse_grained_vorticity! (src/BiotSavart/longrange/longrange.jl:160-186, 273-293): multiply
 * the held coefficients in place by exp(-k^2 * factor), factor = (l^2 - l_old^2) / 2.  With
 * `project` (the reference's cache holds the velocity, whose curl i k x v_k is filtered) the
 * solenoidal part w_k - k (k . w_k) / k^2 is filtered instead (0 at k = 0).  Synchronous. */
int vpbs_coarse_grain(vpbs_handle* h, double factor, int32_t project);

/* interpolate_to_physical! with the default callback (longrange.jl:360-378) followed by
 * copy_long_range_output!: the type-2 NUFFT at the current nodes, with no Ewald filter, of
 * quantity 1 = the held (possibly coarse-grained) vorticity, 2 = the streamfunction w_k / k^2,
 * 3 = the velocity i k x w_k / k^2.  out_xyz: host AoS [Np][3].  Synchronous. */
int vpbs_interpolate_field(vpbs_handle* h, int32_t quantity, double* out_xyz);

/* ---- Time stepping and ensembles (the batching form) ---- */

/* One classic RK4 step (src/Timestepping/timesteppers/explicit/RK4.jl:14-44, advection of
 * advect.jl:40-76) of the filaments last loaded with vpbs_set_filaments: `nodes` is a device AoS
 * array [Np][3] with that filament layout, advanced in place by dt.  Each stage re-solves the
 * splines on the stage nodes with the knots of the first stage (update_coefficients! with
 * knots = ts_base) and evaluates the velocity as vpbs_compute(VELOCITY, LIA_TRUE, both ranges).
 * The velocity of the last stage stays in the handle.  After the first call on a handle it
 * neither allocates nor synchronises with the host (capturable).  Asynchronous on the handle's
 * stream. */
int vpbs_rk4_step(vpbs_handle* h, double* nodes, double dt);

/* An ensemble of independent systems (handles on one device, each holding filaments and its own
 * device node array and time step) advanced together: one RK4 step of every system, each on its
 * own stream, is captured into one CUDA graph at creation (after a dt = 0 warm-up step that
 * leaves the nodes unchanged) and vpbs_ensemble_step replays it `nsteps` times (one graph launch
 * per step, asynchronous on the ensemble's stream).  Errors: vpbs_ensemble_last_error. */
typedef struct vpbs_ensemble vpbs_ensemble;
int vpbs_ensemble_create(vpbs_handle* const* systems, double* const* nodes, const double* dts, int32_t n,
                         vpbs_ensemble** out);
int vpbs_ensemble_step(vpbs_ensemble* e, int32_t nsteps);
int vpbs_ensemble_synchronize(vpbs_ensemble* e);
void* vpbs_ensemble_stream(vpbs_ensemble* e);
int vpbs_ensemble_destroy(vpbs_ensemble* e);
const char* vpbs_ensemble_last_error(void);

/* Autotuner: times the pair kernel on the handle's current point data for each candidate
 * number of cells per CTA edge (1-4, and the built-in rule) and keeps the fastest for later
 * evaluations (`chosen`: 0 = the rule, else the edge).  Overwrites the handle's output fields.
 * Synchronous. */
int vpbs_autotune(vpbs_handle* h, int32_t* chosen);

/* Autotuner of the long range: times one long-range evaluation (spreading, FFTs, Fourier operators,
 * interpolation) on the handle's current point data with each spreading mode of vpbs_spread_mode and
 * keeps the fastest (`chosen`: the mode; mode 0 unless mode 1 is more than 3 % faster).  Overwrites
 * the handle's output fields.  Synchronous. */
int vpbs_autotune_spread(vpbs_handle* h, int32_t* chosen);

/* Spreading kernels of the FP32 (mixed) form for NUFFT half-supports m <= 4 on grids of 16^3 bricks:
 * mode 0 (default) multiplies each brick on the tensor cores (tcgen05, 3xTF32); mode 1 uses the CUDA
 * cores only (plane-owner kernel).  Tuning and testing support; no counterpart in the reference. */
int vpbs_spread_mode(vpbs_handle* h, int32_t mode);

/* Sets the pair kernel's cells per CTA edge for later evaluations (0: the built-in rule; an edge
 * whose neighbourhood does not fit the kernel's tables falls back to the rule), as vpbs_autotune
 * does with its choice.  Tuning support; no counterpart in the reference. */
int vpbs_pair_block(vpbs_handle* h, int32_t cells);

/* ---- Learned parameter predictor (no counterpart in the reference, which removed its alpha
 * autotuner; the fallback is the default rule of splitting/gaussian.jl:133-200). ---- */

/* Features of the configuration loaded in `h` (after vpbs_set_filaments / vpbs_set_points; needs
 * a periodic domain with cell lists): log10 N, log10(line length / L^2), log10(mean and min
 * segment chord / L), and a 12-bin histogram over log10(d / L) in [-3, 0) of the distance d from
 * sampled nodes to their nearest non-local quadrature point (searched within r_cut).  Synchronous. */
#define VPBS_NUM_FEATURES 16
int vpbs_features(vpbs_handle* h, float* out, int32_t n);

/* The predictor network: VPBS_MLP_IN -> VPBS_MLP_HIDDEN -> VPBS_MLP_HIDDEN -> VPBS_MLP_OUT, GELU
 * hidden activations, FP32.  Parameters are one flat array [W1 (H x IN, row-major), b1, W2 (H x H),
 * b2, W3 (OUT x H), b3].  Inputs X are row-major [n][IN], targets and outputs [n][OUT].  The loss
 * is sum_o w_o (y_o - t_o)^2 averaged over the batch (w: vpbs_mlp_set_loss_weights, default 1).
 * vpbs_mlp_train_step runs forward, backward and one Adam step (beta1 0.9, beta2 0.999, eps 1e-8)
 * on the device (with the L2 term of vpbs_mlp_set_weight_decay, default 0); vpbs_mlp_gradient returns
 * the data loss and its gradient without updating.  n must not
 * exceed the max_batch given at creation.  Errors: vpbs_mlp_last_error. */
#define VPBS_MLP_IN 16
#define VPBS_MLP_HIDDEN 64
#define VPBS_MLP_OUT 5
#define VPBS_MLP_NPARAMS (VPBS_MLP_HIDDEN * VPBS_MLP_IN + VPBS_MLP_HIDDEN + VPBS_MLP_HIDDEN * VPBS_MLP_HIDDEN + \
                          VPBS_MLP_HIDDEN + VPBS_MLP_OUT * VPBS_MLP_HIDDEN + VPBS_MLP_OUT)
typedef struct vpbs_mlp vpbs_mlp;
int vpbs_mlp_create(int32_t device, int32_t max_batch, vpbs_mlp** out);
int vpbs_mlp_destroy(vpbs_mlp* m);
const char* vpbs_mlp_last_error(const vpbs_mlp* m);
int vpbs_mlp_set_params(vpbs_mlp* m, const float* params, int64_t n);
int vpbs_mlp_get_params(vpbs_mlp* m, float* params, int64_t n);
int vpbs_mlp_set_loss_weights(vpbs_mlp* m, const float* w);
int vpbs_mlp_set_weight_decay(vpbs_mlp* m, float wd);  /* L2 term (wd/2)|p|^2 in the training loss */
int vpbs_mlp_forward(vpbs_mlp* m, const float* X, int32_t n, float* Y);
int vpbs_mlp_gradient(vpbs_mlp* m, const float* X, const float* T, int32_t n, float* grad, float* loss);
int vpbs_mlp_train_step(vpbs_mlp* m, const float* X, const float* T, int32_t n, float lr, float* loss);

#ifdef __cplusplus
}
#endif
#endif
