// Time stepping of filament systems on the device (the batching form):
//  * vpbs_rk4_step: one classic RK4 step of the filament nodes (src/Timestepping/timesteppers/
//    explicit/RK4.jl:14-44 with the advection of advect.jl:40-76): every stage re-solves the
//    splines on the stage nodes with the knots of the step's first stage (update_coefficients!
//    with knots = ts_base) and evaluates the velocity (LIA, short and long range); no host
//    synchronisation or allocation after the first call, so a step can be captured in a graph;
//  * vpbs_ensemble_*: independent systems advanced together, each on its own stream; one RK4
//    step of every system is captured in one CUDA graph and replayed with one launch per step;
//  * vpbs_autotune: picks the pair kernel's cells per CTA edge by timing the candidates.
#include <string>
#include <vector>

#include "vpbs_internal.cuh"

namespace vpbs {
namespace {

// v: SoA [3][Np] velocity; base, vs, out: AoS [Np][3].
//   mode 0: vs = v;       out = base + a v
//   mode 1: vs += 2 v;    out = base + a v
//   mode 2: base += a (vs + v)
__global__ void rk_update_kernel(int64_t Np, int mode, double a, const double* __restrict__ v, double* base,
                                 double* __restrict__ vs, double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * Np) return;
    const int64_t node = i / 3;
    const int d = (int)(i % 3);
    const double vi = v[d * Np + node];
    if (mode == 0) {
        vs[i] = vi;
        out[i] = base[i] + a * vi;
    } else if (mode == 1) {
        vs[i] += 2.0 * vi;
        out[i] = base[i] + a * vi;
    } else {
        base[i] += a * (vs[i] + vi);
    }
}

}  // namespace
}  // namespace vpbs

using namespace vpbs;

extern "C" int vpbs_rk4_step(vpbs_handle* h, double* nodes, double dt) {
    if (!h || !nodes) return VPBS_ERR_ARG;
    if (!h->have_filaments)
        return set_error(h, VPBS_ERR_STATE, "vpbs_rk4_step needs the filament layout of vpbs_set_filaments");
    int rc;
    if ((rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice"))) return rc;
    const int64_t Np = h->Np;
    if ((rc = ensure(h, h->rk_vs, sizeof(double) * 3 * Np, "RK4 velocity sum"))) return rc;
    if ((rc = ensure(h, h->rk_tmp, sizeof(double) * 3 * Np, "RK4 stage nodes"))) return rc;
    double* vs = (double*)h->rk_vs.p;
    double* tmp = (double*)h->rk_tmp.p;
    const int64_t* offs = (const int64_t*)h->offsets.p;
    const double a[4] = {0.5 * dt, 0.5 * dt, dt, dt / 6.0};
    const double* stage_nodes = nodes;
    for (int s = 0; s < 4; ++s) {
        if ((rc = geometry_from_filaments(h, h->nfil, offs, stage_nodes, h->nmax, s > 0))) return rc;
        h->li_valid = h->K.lia_fraction > 0;
        if ((rc = process_point_charges(h))) return rc;
        if ((rc = vpbs_compute(h, VPBS_VELOCITY, VPBS_LIA_TRUE, 1, 1, 0.0))) return rc;
        const int mode = s == 0 ? 0 : (s < 3 ? 1 : 2);
        rk_update_kernel<<<grid_for(3 * Np, 256), 256, 0, h->stream>>>(Np, mode, a[s], (const double*)h->vel.p, nodes,
                                                                      vs, tmp);
        h->launches++;
        if ((rc = check_cuda(h, cudaGetLastError(), "RK4 update kernel"))) return rc;
        stage_nodes = tmp;
    }
    return 0;
}

struct vpbs_ensemble {
    std::vector<vpbs_handle*> sys;
    std::vector<double*> nodes;
    std::vector<double> dts;
    int device = 0;
    cudaStream_t origin = nullptr;
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_join;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t steps = 0;
};

namespace {
thread_local std::string g_ens_error;

int ens_fail(vpbs_ensemble* e, int code, const std::string& msg) {
    g_ens_error = msg;
    (void)e;
    return code;
}

int ens_cuda(vpbs_ensemble* e, cudaError_t err, const char* what) {
    if (err == cudaSuccess) return 0;
    return ens_fail(e, VPBS_ERR_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(err));
}
}  // namespace

extern "C" {

const char* vpbs_ensemble_last_error(void) { return g_ens_error.c_str(); }

int vpbs_ensemble_destroy(vpbs_ensemble* e) {
    if (!e) return 0;
    cudaSetDevice(e->device);
    if (e->origin) cudaStreamSynchronize(e->origin);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    for (cudaEvent_t ev : e->ev_join)
        if (ev) cudaEventDestroy(ev);
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->origin) cudaStreamDestroy(e->origin);
    delete e;
    return 0;
}

int vpbs_ensemble_create(vpbs_handle* const* systems, double* const* nodes, const double* dts, int32_t n,
                         vpbs_ensemble** out) {
    if (!systems || !nodes || !dts || !out || n < 1) return ens_fail(nullptr, VPBS_ERR_ARG, "bad ensemble arguments");
    *out = nullptr;
    vpbs_ensemble* e = new vpbs_ensemble();
    e->device = systems[0]->device;
    for (int k = 0; k < n; ++k) {
        if (!systems[k] || !nodes[k] || systems[k]->device != e->device || !systems[k]->have_filaments || systems[k]->timing) {
            vpbs_ensemble_destroy(e);
            return ens_fail(nullptr, VPBS_ERR_ARG,
                            "ensemble systems must share one device, hold filaments and have stage timing off");
        }
        e->sys.push_back(systems[k]);
        e->nodes.push_back(nodes[k]);
        e->dts.push_back(dts[k]);
    }
    int rc = ens_cuda(e, cudaSetDevice(e->device), "cudaSetDevice");
    if (!rc) rc = ens_cuda(e, cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!rc) rc = ens_cuda(e, cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming), "cudaEventCreate");
    e->ev_join.assign(n, nullptr);
    for (int k = 0; k < n && !rc; ++k)
        rc = ens_cuda(e, cudaEventCreateWithFlags(&e->ev_join[k], cudaEventDisableTiming), "cudaEventCreate");
    // warm-up step with dt = 0 (nodes unchanged): every buffer, plan and attribute is in place
    // before the capture
    for (int k = 0; k < n && !rc; ++k)
        if (vpbs_rk4_step(e->sys[k], e->nodes[k], 0.0)) rc = ens_fail(e, VPBS_ERR_CUDA, vpbs_last_error(e->sys[k]));
    if (!rc) rc = ens_cuda(e, cudaDeviceSynchronize(), "warm-up");
    if (!rc) rc = ens_cuda(e, cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeRelaxed), "begin capture");
    if (!rc) {
        int crc = ens_cuda(e, cudaEventRecord(e->ev_fork, e->origin), "fork");
        for (int k = 0; k < n && !crc; ++k) {
            vpbs_handle* h = e->sys[k];
            crc = ens_cuda(e, cudaStreamWaitEvent(h->stream, e->ev_fork, 0), "fork");
            if (!crc && vpbs_rk4_step(h, e->nodes[k], e->dts[k])) crc = ens_fail(e, VPBS_ERR_CUDA, vpbs_last_error(h));
            if (!crc) crc = ens_cuda(e, cudaEventRecord(e->ev_join[k], h->stream), "join");
            if (!crc) crc = ens_cuda(e, cudaStreamWaitEvent(e->origin, e->ev_join[k], 0), "join");
        }
        const cudaError_t end = cudaStreamEndCapture(e->origin, &e->graph);
        rc = crc ? crc : ens_cuda(e, end, "end capture");
    }
    if (!rc) rc = ens_cuda(e, cudaGraphInstantiate(&e->exec, e->graph, 0), "graph instantiate");
    if (rc) {
        vpbs_ensemble_destroy(e);
        return rc;
    }
    *out = e;
    return 0;
}

int vpbs_ensemble_step(vpbs_ensemble* e, int32_t nsteps) {
    if (!e || nsteps < 0) return ens_fail(e, VPBS_ERR_ARG, "bad ensemble step arguments");
    int rc = ens_cuda(e, cudaSetDevice(e->device), "cudaSetDevice");
    for (int s = 0; s < nsteps && !rc; ++s) rc = ens_cuda(e, cudaGraphLaunch(e->exec, e->origin), "graph launch");
    if (!rc) e->steps += nsteps;
    return rc;
}

int vpbs_ensemble_synchronize(vpbs_ensemble* e) {
    if (!e) return VPBS_ERR_ARG;
    int rc = ens_cuda(e, cudaSetDevice(e->device), "cudaSetDevice");
    if (!rc) rc = ens_cuda(e, cudaStreamSynchronize(e->origin), "synchronize");
    return rc;
}

void* vpbs_ensemble_stream(vpbs_ensemble* e) { return e ? (void*)e->origin : nullptr; }

int vpbs_autotune(vpbs_handle* h, int32_t* chosen) {
    if (!h) return VPBS_ERR_ARG;
    if (!h->have_points) return set_error(h, VPBS_ERR_STATE, "vpbs_autotune needs point data");
    if (h->K.open_domain || h->cg.M < 1) {
        if (chosen) *chosen = 0;
        return 0;  // no cell lists: nothing to tune
    }
    int rc;
    if ((rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice"))) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const bool timing = h->timing;
    h->timing = false;
    float best = 1e30f;
    int best_b = 0;
    for (int b = 0; b <= 4 && !rc; ++b) {  // b = 0: the built-in rule
        h->pair_block = b;
        float tmin = 1e30f;
        for (int rep = 0; rep < 3 && !rc; ++rep) {
            cudaEventRecord(e0, h->stream);
            rc = pair_interactions(h, VPBS_VELOCITY);
            cudaEventRecord(e1, h->stream);
            if (!rc) rc = check_cuda(h, cudaEventSynchronize(e1), "autotune sync");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tmin = fminf(tmin, ms);
        }
        if (!rc && tmin < best * 0.97f) {  // keep the simpler choice unless clearly faster
            best = tmin;
            best_b = b;
        }
    }
    h->pair_block = best_b;
    h->timing = timing;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (chosen) *chosen = best_b;
    return rc;
}

int vpbs_autotune_spread(vpbs_handle* h, int32_t* chosen) {
    if (!h) return VPBS_ERR_ARG;
    if (!h->have_points) return set_error(h, VPBS_ERR_STATE, "vpbs_autotune_spread needs point data");
    if (h->K.open_domain) {
        if (chosen) *chosen = h->spread_mode;
        return 0;  // no long range: nothing to tune
    }
    int rc;
    if ((rc = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice"))) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const bool timing = h->timing;
    h->timing = false;
    float best = 1e30f;
    int best_m = 0;
    for (int mode = 0; mode <= 1 && !rc; ++mode) {  // mode 0: the default
        h->spread_mode = mode;
        float tmin = 1e30f;
        for (int rep = 0; rep < 3 && !rc; ++rep) {
            cudaEventRecord(e0, h->stream);
            rc = longrange_compute(h, VPBS_VELOCITY);
            cudaEventRecord(e1, h->stream);
            if (!rc) rc = check_cuda(h, cudaEventSynchronize(e1), "autotune sync");
            if (!rc) rc = check_status(h);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tmin = fminf(tmin, ms);
        }
        if (!rc && tmin < best * 0.97f) {  // keep the default unless the other is clearly faster
            best = tmin;
            best_m = mode;
        }
    }
    h->spread_mode = best_m;
    h->timing = timing;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (chosen) *chosen = best_m;
    return rc;
}

int vpbs_pair_block(vpbs_handle* h, int32_t cells) {
    if (!h || cells < 0 || cells > 8) return VPBS_ERR_ARG;
    h->pair_block = cells;
    return 0;
}

}  // extern "C"
