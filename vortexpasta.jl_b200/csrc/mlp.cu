// Parameter predictor network: a 16 -> 64 -> 64 -> 5 multilayer perceptron with GELU
// activations, in FP32, with hand-written forward, backward and Adam kernels.  It maps cheap
// features of a filament configuration to Ewald/NUFFT parameters (the library's own sweeps
// provide the training targets).  The layers are tiny, so every kernel is a plain
// one-thread-per-output loop over the reduction dimension; the weights live in one flat
// device buffer [W1 (64x16), b1, W2 (64x64), b2, W3 (5x64), b3].
#include <cmath>
#include <new>
#include <string>

#include "vpbs_internal.cuh"

namespace {

constexpr int kIn = VPBS_MLP_IN, kHid = VPBS_MLP_HIDDEN, kOut = VPBS_MLP_OUT;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kOut * kHid, kNParams = kOffB3 + kOut;
static_assert(kNParams == VPBS_MLP_NPARAMS, "parameter count");

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
// d/dz [z Phi(z)] = Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Z[n][o] = b[o] + sum_i W[o][i] X[n][i];  H = gelu(Z) when act.
__global__ void dense_forward_kernel(int n, int nin, int nout, const float* __restrict__ X, const float* __restrict__ W,
                                     const float* __restrict__ b, float* __restrict__ Z, float* __restrict__ H, int act) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * nout) return;
    const int r = idx / nout, o = idx % nout;
    float s = b[o];
    const float* x = X + (size_t)r * nin;
    const float* w = W + (size_t)o * nin;
    for (int i = 0; i < nin; ++i) s = fmaf(w[i], x[i], s);
    Z[idx] = s;
    if (H) H[idx] = act ? gelu(s) : s;
}

// dY = wts (Y - T) 2 / n, and the loss sum_n sum_o wts_o (Y - T)^2 / n (atomic).
__global__ void loss_grad_kernel(int n, const float* __restrict__ Y, const float* __restrict__ T,
                                 const float* __restrict__ wts, float* __restrict__ dY, float* __restrict__ loss) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * kOut) return;
    const int o = idx % kOut;
    const float d = Y[idx] - T[idx];
    dY[idx] = 2.0f * wts[o] * d / n;
    atomicAdd(loss, wts[o] * d * d / n);
}

// dW[o][i] = sum_r dZ[r][o] X[r][i];  db[o] = sum_r dZ[r][o]  (one thread per weight).
__global__ void dense_weight_grad_kernel(int n, int nin, int nout, const float* __restrict__ X,
                                         const float* __restrict__ dZ, float* __restrict__ dW, float* __restrict__ db) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nout * (nin + 1)) return;
    const int o = idx / (nin + 1), i = idx % (nin + 1);
    float s = 0.0f;
    if (i < nin)
        for (int r = 0; r < n; ++r) s = fmaf(dZ[(size_t)r * nout + o], X[(size_t)r * nin + i], s);
    else
        for (int r = 0; r < n; ++r) s += dZ[(size_t)r * nout + o];
    if (i < nin) dW[(size_t)o * nin + i] = s;
    else db[o] = s;
}

// dZprev[r][i] = gelu'(Zprev[r][i]) sum_o W[o][i] dZ[r][o]
__global__ void dense_input_grad_kernel(int n, int nin, int nout, const float* __restrict__ W,
                                        const float* __restrict__ dZ, const float* __restrict__ Zprev,
                                        float* __restrict__ dZprev) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * nin) return;
    const int r = idx / nin, i = idx % nin;
    float s = 0.0f;
    for (int o = 0; o < nout; ++o) s = fmaf(W[(size_t)o * nin + i], dZ[(size_t)r * nout + o], s);
    dZprev[idx] = s * gelu_grad(Zprev[idx]);
}

// Adam (Kingma & Ba 2015) with bias correction on the loss plus (wd/2)|p|^2; step t >= 1.
__global__ void adam_kernel(int np, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2,
                            float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float gi = g[i] + wd * p[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    p[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

inline unsigned nblk(int n) { return (unsigned)((n + 255) / 256); }

}  // namespace

struct vpbs_mlp {
    int device = 0;
    int max_batch = 0;
    int64_t steps = 0;
    float weight_decay = 0.0f;
    std::string err;
    cudaStream_t stream = nullptr;
    float* params = nullptr;  // kNParams
    float* grad = nullptr;    // kNParams
    float* m1 = nullptr;
    float* m2 = nullptr;
    float* X = nullptr;  // max_batch x kIn
    float* T = nullptr;  // max_batch x kOut
    float* wts = nullptr;  // kOut
    float* Z1 = nullptr; float* H1 = nullptr;
    float* Z2 = nullptr; float* H2 = nullptr;
    float* Y = nullptr;
    float* dY = nullptr; float* dZ2 = nullptr; float* dZ1 = nullptr;
    float* loss = nullptr;
};

namespace {

int mlp_err(vpbs_mlp* m, int code, const std::string& msg) {
    if (m) m->err = msg;
    return code;
}

int mlp_cuda(vpbs_mlp* m, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return 0;
    return mlp_err(m, VPBS_ERR_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

int mlp_forward_device(vpbs_mlp* m, int n) {
    const float* P = m->params;
    dense_forward_kernel<<<nblk(n * kHid), 256, 0, m->stream>>>(n, kIn, kHid, m->X, P + kOffW1, P + kOffB1, m->Z1, m->H1, 1);
    dense_forward_kernel<<<nblk(n * kHid), 256, 0, m->stream>>>(n, kHid, kHid, m->H1, P + kOffW2, P + kOffB2, m->Z2, m->H2,
                                                                1);
    dense_forward_kernel<<<nblk(n * kOut), 256, 0, m->stream>>>(n, kHid, kOut, m->H2, P + kOffW3, P + kOffB3, m->Y,
                                                                nullptr, 0);
    return mlp_cuda(m, cudaGetLastError(), "MLP forward");
}

// loss and gradient for the batch already in m->X / m->T
int mlp_backward_device(vpbs_mlp* m, int n) {
    int rc;
    if ((rc = mlp_forward_device(m, n))) return rc;
    float* G = m->grad;
    const float* P = m->params;
    if ((rc = mlp_cuda(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream), "memset"))) return rc;
    loss_grad_kernel<<<nblk(n * kOut), 256, 0, m->stream>>>(n, m->Y, m->T, m->wts, m->dY, m->loss);
    dense_weight_grad_kernel<<<nblk(kOut * (kHid + 1)), 256, 0, m->stream>>>(n, kHid, kOut, m->H2, m->dY, G + kOffW3,
                                                                             G + kOffB3);
    dense_input_grad_kernel<<<nblk(n * kHid), 256, 0, m->stream>>>(n, kHid, kOut, P + kOffW3, m->dY, m->Z2, m->dZ2);
    dense_weight_grad_kernel<<<nblk(kHid * (kHid + 1)), 256, 0, m->stream>>>(n, kHid, kHid, m->H1, m->dZ2, G + kOffW2,
                                                                             G + kOffB2);
    dense_input_grad_kernel<<<nblk(n * kHid), 256, 0, m->stream>>>(n, kHid, kHid, P + kOffW2, m->dZ2, m->Z1, m->dZ1);
    dense_weight_grad_kernel<<<nblk(kHid * (kIn + 1)), 256, 0, m->stream>>>(n, kIn, kHid, m->X, m->dZ1, G + kOffW1,
                                                                            G + kOffB1);
    return mlp_cuda(m, cudaGetLastError(), "MLP backward");
}

int mlp_upload_batch(vpbs_mlp* m, const float* X, const float* T, int n) {
    if (n < 1 || n > m->max_batch) return mlp_err(m, VPBS_ERR_ARG, "batch size out of range");
    int rc;
    if ((rc = mlp_cuda(m, cudaMemcpyAsync(m->X, X, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, m->stream), "copy X")))
        return rc;
    if (T && (rc = mlp_cuda(m, cudaMemcpyAsync(m->T, T, sizeof(float) * n * kOut, cudaMemcpyHostToDevice, m->stream),
                            "copy T")))
        return rc;
    return 0;
}

}  // namespace

extern "C" {

int vpbs_mlp_create(int32_t device, int32_t max_batch, vpbs_mlp** out) {
    if (!out || max_batch < 1) return VPBS_ERR_ARG;
    *out = nullptr;
    vpbs_mlp* m = new (std::nothrow) vpbs_mlp();
    if (!m) return VPBS_ERR_OOM;
    m->device = device;
    m->max_batch = max_batch;
    int rc = mlp_cuda(m, cudaSetDevice(device), "cudaSetDevice");
    if (!rc) rc = mlp_cuda(m, cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    const size_t nb = (size_t)max_batch;
    float** bufs[] = {&m->params, &m->grad, &m->m1, &m->m2, &m->X, &m->T, &m->wts, &m->Z1, &m->H1,
                      &m->Z2, &m->H2, &m->Y, &m->dY, &m->dZ2, &m->dZ1, &m->loss};
    const size_t sizes[] = {kNParams, kNParams, kNParams, kNParams, nb * kIn, nb * kOut, kOut, nb * kHid, nb * kHid,
                            nb * kHid, nb * kHid, nb * kOut, nb * kOut, nb * kHid, nb * kHid, 1};
    for (int i = 0; i < 16 && !rc; ++i) rc = mlp_cuda(m, cudaMalloc(bufs[i], sizeof(float) * sizes[i]), "cudaMalloc");
    if (!rc) rc = mlp_cuda(m, cudaMemset(m->params, 0, sizeof(float) * kNParams), "memset");
    if (!rc) rc = mlp_cuda(m, cudaMemset(m->m1, 0, sizeof(float) * kNParams), "memset");
    if (!rc) rc = mlp_cuda(m, cudaMemset(m->m2, 0, sizeof(float) * kNParams), "memset");
    if (!rc) {
        const float ones[kOut] = {1, 1, 1, 1, 1};
        rc = mlp_cuda(m, cudaMemcpy(m->wts, ones, sizeof(ones), cudaMemcpyHostToDevice), "copy");
    }
    if (rc) {
        vpbs_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return 0;
}

int vpbs_mlp_destroy(vpbs_mlp* m) {
    if (!m) return 0;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    float* bufs[] = {m->params, m->grad, m->m1, m->m2, m->X, m->T, m->wts, m->Z1, m->H1,
                     m->Z2, m->H2, m->Y, m->dY, m->dZ2, m->dZ1, m->loss};
    for (float* b : bufs)
        if (b) cudaFree(b);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return 0;
}

const char* vpbs_mlp_last_error(const vpbs_mlp* m) { return m ? m->err.c_str() : ""; }

int vpbs_mlp_set_params(vpbs_mlp* m, const float* params, int64_t n) {
    if (!m || !params || n != kNParams) return mlp_err(m, VPBS_ERR_ARG, "expected VPBS_MLP_NPARAMS parameters");
    int rc = mlp_cuda(m, cudaSetDevice(m->device), "cudaSetDevice");
    if (!rc) rc = mlp_cuda(m, cudaMemcpy(m->params, params, sizeof(float) * kNParams, cudaMemcpyHostToDevice), "copy");
    if (!rc) rc = mlp_cuda(m, cudaMemset(m->m1, 0, sizeof(float) * kNParams), "memset");
    if (!rc) rc = mlp_cuda(m, cudaMemset(m->m2, 0, sizeof(float) * kNParams), "memset");
    m->steps = 0;
    return rc;
}

int vpbs_mlp_get_params(vpbs_mlp* m, float* params, int64_t n) {
    if (!m || !params || n != kNParams) return mlp_err(m, VPBS_ERR_ARG, "expected VPBS_MLP_NPARAMS parameters");
    int rc = mlp_cuda(m, cudaSetDevice(m->device), "cudaSetDevice");
    if (!rc) rc = mlp_cuda(m, cudaStreamSynchronize(m->stream), "sync");
    if (!rc) rc = mlp_cuda(m, cudaMemcpy(params, m->params, sizeof(float) * kNParams, cudaMemcpyDeviceToHost), "copy");
    return rc;
}

int vpbs_mlp_set_loss_weights(vpbs_mlp* m, const float* w) {
    if (!m || !w) return VPBS_ERR_ARG;
    int rc = mlp_cuda(m, cudaSetDevice(m->device), "cudaSetDevice");
    if (!rc) rc = mlp_cuda(m, cudaMemcpy(m->wts, w, sizeof(float) * kOut, cudaMemcpyHostToDevice), "copy");
    return rc;
}

int vpbs_mlp_set_weight_decay(vpbs_mlp* m, float wd) {
    if (!m || !(wd >= 0.0f)) return mlp_err(m, VPBS_ERR_ARG, "weight decay must be >= 0");
    m->weight_decay = wd;
    return 0;
}

int vpbs_mlp_forward(vpbs_mlp* m, const float* X, int32_t n, float* Y) {
    if (!m || !X || !Y) return VPBS_ERR_ARG;
    int rc = mlp_cuda(m, cudaSetDevice(m->device), "cudaSetDevice");
    if (!rc) rc = mlp_upload_batch(m, X, nullptr, n);
    if (!rc) rc = mlp_forward_device(m, n);
    if (!rc) rc = mlp_cuda(m, cudaMemcpyAsync(Y, m->Y, sizeof(float) * n * kOut, cudaMemcpyDeviceToHost, m->stream), "copy Y");
    if (!rc) rc = mlp_cuda(m, cudaStreamSynchronize(m->stream), "sync");
    return rc;
}

int vpbs_mlp_gradient(vpbs_mlp* m, const float* X, const float* T, int32_t n, float* grad, float* loss) {
    if (!m || !X || !T || !grad || !loss) return VPBS_ERR_ARG;
    int rc = mlp_cuda(m, cudaSetDevice(m->device), "cudaSetDevice");
    if (!rc) rc = mlp_upload_batch(m, X, T, n);
    if (!rc) rc = mlp_backward_device(m, n);
    if (!rc) rc = mlp_cuda(m, cudaMemcpyAsync(grad, m->grad, sizeof(float) * kNParams, cudaMemcpyDeviceToHost, m->stream),
                           "copy grad");
    if (!rc) rc = mlp_cuda(m, cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream), "copy loss");
    if (!rc) rc = mlp_cuda(m, cudaStreamSynchronize(m->stream), "sync");
    return rc;
}

int vpbs_mlp_train_step(vpbs_mlp* m, const float* X, const float* T, int32_t n, float lr, float* loss) {
    if (!m || !X || !T) return VPBS_ERR_ARG;
    int rc = mlp_cuda(m, cudaSetDevice(m->device), "cudaSetDevice");
    if (!rc) rc = mlp_upload_batch(m, X, T, n);
    if (!rc) rc = mlp_backward_device(m, n);
    if (rc) return rc;
    m->steps++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)m->steps), c2 = 1.0f - std::pow(b2, (float)m->steps);
    adam_kernel<<<nblk(kNParams), 256, 0, m->stream>>>(kNParams, m->params, m->grad, m->m1, m->m2, lr, b1, b2, 1e-8f,
                                                       c1, c2, m->weight_decay);
    rc = mlp_cuda(m, cudaGetLastError(), "Adam kernel");
    if (!rc && loss) {
        rc = mlp_cuda(m, cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream), "copy loss");
        if (!rc) rc = mlp_cuda(m, cudaStreamSynchronize(m->stream), "sync");
    }
    return rc;
}

}  // extern "C"
