// Internal declarations shared by the libvpbs.so translation units.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <string>
#include <vector>

#include "vpbs.h"

namespace vpbs {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxQuad = 16;
constexpr int kMaxHalfSupport = 8;

// Parameters in the form the kernels use (passed by value to kernels).
struct KParams {
    double Gamma, a, Delta;
    double L[3], Lh[3];
    double alpha, rcut, rcut2;
    int nquad, nquad_near;
    double qz[kMaxQuad], qw[kMaxQuad];
    double qnz[kMaxQuad], qnw[kMaxQuad];
    double lia_fraction;  // <= 0: nothing
    int avoid_explicit_erf;
    int open_domain;      // NoSplitting
    int kb;               // KaiserBesselSplitting: the long-range weights vanish beyond rcut
    // piecewise Taylor tables of erfc(x) and erfc(x) + 2/sqrt(pi) x exp(-x^2), x = alpha r
    const double* ewald_tab;
    const float* ewald_tab_f;  // FP32 copy (first kEwaldNCf coefficients) for the mixed form
    const double2* ewald_tab2; // interleaved (erfc, g) coefficient pairs, for both weights at once
    int ewald_ntab;       // number of intervals (0: no splitting, weights are 1)
    // FP32 cubic tables of the mixed form's pair kernel: intervals of width 1/32 in x, one float4
    // (c0, c1, c2, c3) in powers of t = 32 x - k per interval k; weight a then weight g
    const float4* tab_c;
    int ntab_c;
};

// Ewald weight tables: intervals of width 1/16 in x = alpha r, degree-9 Taylor polynomials
// about the interval centres (coefficients from the closed-form derivatives of erfc).
constexpr int kEwaldNC = 10;
constexpr int kEwaldNCf = 6;  // FP32 tables: degree 5 (remainder < 1e-9 on |x - c| <= 1/32)
constexpr double kEwaldInvH = 16.0;
constexpr double kEwaldH = 1.0 / 16.0;
void ewald_table_host(double xmax, int* ntab, double* tab);  // tab: 2 * ntab * kEwaldNC doubles
int ewald_table_size(double xmax);
// Both weights from a table in the layout of ewald_table_host (host evaluation, FP64).
void table_eval_host(const double* tab, int ntab, double x, double* a, double* g);
// FP32 cubic tables fitted to an FP64 table over [0, xmax] (layout of KParams::tab_c): nf intervals.
constexpr float kTabCInvH = 32.0f;
int f32_table_size(double xmax);
void f32_table_host(const double* tab, int ntab, double xmax, float4* out);  // out: 2 * f32_table_size(xmax)
// Device-identical host evaluation of the FP32 cubic tables (same float operations).
void f32_table_eval_host(const float4* tabc, int nf, float x, float* a, float* g);

// Gauss-Legendre rule on [-1, 1] (host; longrange.cu).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);

// Kaiser-Bessel splitting (splitting.cu): the reference's truncated Chebyshev series of the kernel
// f and of its integral F (full coefficient vectors in u = r / rcut), and their weight tables in
// the layout of ewald_table_host over x = (kb_table_xmax(beta) / rcut) r.
struct KBSeries {
    double beta = 0.0, rcut = 0.0;
    std::vector<double> f, F;
};
KBSeries kb_series(double beta, double rcut, double rtol);
void kb_weights_series(const KBSeries& S, double r, double* a, double* g);
double kb_table_xmax(double beta);
void kb_table_host(const KBSeries& S, int* ntab, double* tab);

__device__ __forceinline__ void ewald_weights(const KParams& K, double x, double& a, double& g) {
    int k = (int)(x * kEwaldInvH);
    k = k < K.ewald_ntab ? k : K.ewald_ntab - 1;
    const double t = x - (k + 0.5) * kEwaldH;
    const double* ce = K.ewald_tab + k * kEwaldNC;
    const double* cg = K.ewald_tab + (K.ewald_ntab + k) * kEwaldNC;
    a = __ldg(ce + kEwaldNC - 1);
    g = __ldg(cg + kEwaldNC - 1);
#pragma unroll
    for (int n = kEwaldNC - 2; n >= 0; --n) {
        a = fma(a, t, __ldg(ce + n));
        g = fma(g, t, __ldg(cg + n));
    }
}

// Rank of this thread's element within its bin, from one atomicAdd per distinct bin in the warp:
// the points arrive in cell order, so the lanes of a warp mostly share a bin, and 32 same-address
// atomics would serialise.  Lanes of the warp that have exited must not be named in the mask.
__device__ __forceinline__ int32_t warp_aggregated_rank(int32_t* counts, int32_t b) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, b);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int32_t base = 0;
    if (lane == leader) base = atomicAdd(&counts[b], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

// Cell-list geometry.  Cells are r_cut / M wide in y and z (M = nsubdiv); in x each such
// cell is further split into G slabs (nc[0] counts the slabs), so the candidate range of a
// node in a row of cells can be trimmed to the slabs within r_cut.
struct CellGrid {
    int nc[3];
    int M;
    int G;
    int64_t ncell;
};

// Long-range sizes.
struct LRSizes {
    int Ns[3];
    int nkx;         // Ns0/2 + 1
    int n[3];        // oversampled FFT grid
    int nxc;         // n0/2 + 1
    int64_t ngrid;   // n0*n1*n2 (real)
    int64_t ncgrid;  // nxc*n1*n2 (complex)
    int64_t nmodes;  // nkx*Ns1*Ns2
    int m;
    double beta;     // spreading-kernel shape
    double edge;     // the kernel's value at |u| = m, subtracted so that it vanishes there
    int kernel;      // VPBS_NUFFT_*
};

// Host <-> device staging of flat node and output arrays goes in chunks of at least
// kStageChunk bytes (at most kStageEvents of them), host copies overlapping the transfers.
constexpr size_t kStageChunk = (size_t)4 << 20;
constexpr int kStageEvents = 16;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace vpbs

struct vpbs_handle {
    vpbs_params P;
    vpbs::KParams K;
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int64_t launches = 0;

    // sizes
    int64_t Np = 0, Nq = 0, nfil = 0;
    bool have_points = false;

    // geometry inputs / scratch
    vpbs::DevBuf nodes_in, offsets, fil_of_node, knots, coefs, dcoef1, dcoef2, spline_scratch;
    // end-to-end offsets of unclosed (infinite) filaments, [nfil][3] (closed_filament.jl:118-132)
    vpbs::DevBuf fil_off;
    bool have_fil_offsets = false;
    double offset_sum[3] = {0.0, 0.0, 0.0};  // sum over the filaments (background vorticity)
    int64_t nfil_off = 0;                     // filament count the offsets were given for
    double bg_factor = 0.0;  // streamfunction of a unit uniform vorticity (background_vorticity_correction_factor)

    // point data (SoA; 3 consecutive blocks of Np or Nq doubles for vectors)
    vpbs::DevBuf nodes, idx_prev, d1, d2, dm, dp, points, charges;
    vpbs::DevBuf li_vel, li_psi;  // lia_segment_fraction local integrals (per node)

    // cell lists
    vpbs::CellGrid cg{};
    vpbs::DevBuf src_cell, src_start, src_fill, src_sorted, src_seg, dst_cell, dst_start, dst_fill, dst_order;
    vpbs::DevBuf counters;  // [0] in-range pairs, [1] candidates (unsigned long long)
    vpbs::DevBuf scan_tmp, scan_tmp_lr;  // multi-CTA scan scratch (cell lists; spreading bins)
    vpbs::DevBuf ewald_tab;  // Taylor tables of the Ewald weights (KParams::ewald_tab)

    // long range
    vpbs::LRSizes lr{};
    vpbs::DevBuf grid_r, grid_c, grid_c2, uhat, decx, decy, decz, nodes_lr;
    vpbs::DevBuf spread_bin, spread_counts, spread_start, binned, spread_foot;  // brick spreading
    vpbs::DevBuf tc_counts, tc_start, tc_rec;  // tensor-core spreading: per-brick (point, brick) records
    vpbs::DevBuf peer_in;                       // vpbs_add_field: a field copied from another GPU
    cudaEvent_t xfer_done = nullptr;            // vpbs_add_field: this handle's fields are complete
    int gatherB = 0;   // brick edge of the atomic-free spreading (0: atomic fallback)
    int spread_mode = 0;  // 0: tensor-core spreading where it applies; 1: CUDA-core kernels only
    int* status_host = nullptr;  // mapped pinned word: device-side faults of bounded waits (0: none)
    int* status_dev = nullptr;
    int nbrick[3] = {0, 0, 0};
    cufftHandle plan_r2c = 0, plan_c2r = 0, plan_c2r_6 = 0;
    bool have_plans = false;
    bool have_uhat = false;

    // outputs (SoA, 3*Np each)
    vpbs::DevBuf vel, psi;
    int32_t last_fields = 0;

    // pinned host staging: separate regions for inputs and outputs; h2d_done guards reuse
    void* pin_in = nullptr;
    size_t pin_in_bytes = 0;
    void* pin_out = nullptr;
    size_t pin_out_bytes = 0;
    cudaEvent_t h2d_done = nullptr;
    bool li_valid = false;  // lia_segment_fraction integrals available (filament input only)

    // the long range runs on aux_stream concurrently with the short range (fork/join events)
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_short = nullptr, ev_long = nullptr;
    cudaEvent_t interp_wait = nullptr;  // event the interpolation waits for (outputs are shared)

    std::vector<int64_t> host_offsets;  // filament layout of the last vpbs_set_filaments (host copy)
    cudaEvent_t stage_ev[vpbs::kStageEvents] = {};  // chunked host <-> device staging
    vpbs::DevBuf aos_out;                 // AoS staging of an output field (vpbs_get_filaments)

    // time stepping (vpbs_rk4_step): filament layout of the last vpbs_set_filaments, RK buffers
    int64_t nmax = 0;
    bool have_filaments = false;
    vpbs::DevBuf rk_vs, rk_tmp;
    // pair-kernel cells per CTA edge chosen by vpbs_autotune (0: the built-in rule)
    int pair_block = 0;

    // optional per-stage CUDA-event timing (vpbs_stage_timing)
    bool timing = false;
    cudaEvent_t tev[16][4][2] = {};  // [stage][occurrence][start/stop]
    int tcount[16] = {};
};

namespace vpbs {

int set_error(vpbs_handle* h, int code, const std::string& msg);
int check_cuda(vpbs_handle* h, cudaError_t e, const char* what);
int ensure(vpbs_handle* h, DevBuf& b, size_t bytes, const char* what);
int ensure_pinned(vpbs_handle* h, void** buf, size_t* cap, size_t bytes);
int ensure_status(vpbs_handle* h);   // the mapped status word of bounded device-side waits
int check_status(vpbs_handle* h);    // after a synchronisation: VPBS_ERR_TIMEOUT if a wait gave up

inline unsigned grid_for(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

// geometry.cu
int geometry_from_filaments(vpbs_handle* h, int64_t nfil, const int64_t* d_offsets, const double* d_nodes,
                            int64_t nmax, bool keep_knots = false);  // nmax: largest node count of a filament

// api.cu
int process_point_charges(vpbs_handle* h);  // cell lists of the current point data
CellGrid make_cell_grid(const double L[3], double rcut, int M);

// shortrange.cu
int build_cell_lists(vpbs_handle* h);
int exclusive_scan(vpbs_handle* h, const int32_t* counts, int32_t* start, int64_t n,
                   DevBuf& tmp);  // start[0..n]; tmp: scratch of the multi-CTA scan
int local_and_self(vpbs_handle* h, int fields, int lia_mode, int with_pairs_self, double integration_cutoff);
int pair_interactions(vpbs_handle* h, int fields);
int add_local_integrals(vpbs_handle* h, int fields);

// longrange.cu
int longrange_init(vpbs_handle* h);
void longrange_free(vpbs_handle* h);
int longrange_compute(vpbs_handle* h, int fields);  // adds into h->vel / h->psi

// stage timing
enum Stage {
    ST_GEOMETRY = 0, ST_CELL_LISTS, ST_SPREAD, ST_FFT_FORWARD, ST_FOURIER, ST_FFT_INVERSE, ST_INTERP,
    ST_LOCAL_SELF, ST_PAIRS, ST_COUNT
};
inline void stage_mark(vpbs_handle* h, int s, int stop) {
    if (!h->timing) return;
    int k = stop ? h->tcount[s] - 1 : h->tcount[s];
    if (k < 0 || k >= 4) return;
    cudaEventRecord(h->tev[s][k][stop], h->stream);
    if (!stop) h->tcount[s]++;
}
struct StageScope {
    vpbs_handle* h;
    int s;
    StageScope(vpbs_handle* hh, int ss) : h(hh), s(ss) { stage_mark(h, s, 0); }
    ~StageScope() { stage_mark(h, s, 1); }
};

}  // namespace vpbs
