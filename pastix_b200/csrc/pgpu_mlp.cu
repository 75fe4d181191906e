// Learned cost model: a small multilayer perceptron (F inputs -> H -> H -> 1,
// ReLU) that predicts the device time of a factorization task from its
// shape.  It replaces the polynomial kernel models of the reference
// (common/models.c: per-kernel polynomials in the block sizes, fitted
// offline) in ordering the work of a level and in sharding independent
// systems over GPUs.  Training and inference run on the GPU with the kernels
// below, in FP64 (the model is tiny; FP64 keeps the gradient check against
// the CPU restatement at rounding level).
//
// Parameters, packed: W1[H][F], b1[H], W2[H][H], b2[H], W3[H], b3.
//   a1 = relu(W1 x + b1), a2 = relu(W2 a1 + b2), y = W3 . a2 + b3
// Loss: mean squared error over the batch, L = (1/n) sum (y_s - t_s)^2.
#include "pastix_gpu.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr int MLP_HMAX = 64;
constexpr int MLP_FMAX = 32;

struct Layout {
    int F, H;
    __host__ __device__ int64_t w1() const { return 0; }
    __host__ __device__ int64_t b1() const { return (int64_t)H * F; }
    __host__ __device__ int64_t w2() const { return b1() + H; }
    __host__ __device__ int64_t b2() const { return w2() + (int64_t)H * H; }
    __host__ __device__ int64_t w3() const { return b2() + H; }
    __host__ __device__ int64_t b3() const { return w3() + H; }
    __host__ __device__ int64_t count() const { return b3() + 1; }
};

// one thread per sample; activations kept for the backward pass
__global__ void k_mlp_forward(int64_t n, Layout L, const double *__restrict__ X, const double *__restrict__ P,
                              double *__restrict__ A1, double *__restrict__ A2, double *__restrict__ Y) {
    const int F = L.F, H = L.H;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        const double *x = X + s * F;
        double a1[MLP_HMAX];
        for (int j = 0; j < H; j++) {
            double v = P[L.b1() + j];
            for (int i = 0; i < F; i++) v += P[L.w1() + (int64_t)j * F + i] * x[i];
            a1[j] = v > 0.0 ? v : 0.0;
            if (A1) A1[s * H + j] = a1[j];
        }
        double y = P[L.b3()];
        for (int k = 0; k < H; k++) {
            double v = P[L.b2() + k];
            for (int j = 0; j < H; j++) v += P[L.w2() + (int64_t)k * H + j] * a1[j];
            v = v > 0.0 ? v : 0.0;
            if (A2) A2[s * H + k] = v;
            y += P[L.w3() + k] * v;
        }
        Y[s] = y;
    }
}

// per-sample output and hidden deltas of the squared-error loss
__global__ void k_mlp_delta(int64_t n, Layout L, const double *__restrict__ P, const double *__restrict__ A1,
                            const double *__restrict__ A2, const double *__restrict__ Y,
                            const double *__restrict__ T, double *__restrict__ DY, double *__restrict__ D2,
                            double *__restrict__ D1) {
    const int H = L.H;
    const double scale = 2.0 / (double)n;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        const double dy = scale * (Y[s] - T[s]);
        DY[s] = dy;
        double d2[MLP_HMAX];
        for (int k = 0; k < H; k++) {
            d2[k] = (A2[s * H + k] > 0.0) ? dy * P[L.w3() + k] : 0.0;
            D2[s * H + k] = d2[k];
        }
        for (int j = 0; j < H; j++) {
            double v = 0.0;
            if (A1[s * H + j] > 0.0)
                for (int k = 0; k < H; k++) v += P[L.w2() + (int64_t)k * H + j] * d2[k];
            D1[s * H + j] = v;
        }
    }
}

// Gradient, in two deterministic passes: chunk c of MLP_CHUNK samples gives
// partial[c][p] (one thread per parameter p, samples in order), then the
// chunks are summed in order.
constexpr int MLP_CHUNK = 1024;

__global__ void k_mlp_grad_partial(int64_t n, Layout L, const double *__restrict__ X, const double *__restrict__ A1,
                                   const double *__restrict__ A2, const double *__restrict__ DY,
                                   const double *__restrict__ D2, const double *__restrict__ D1,
                                   double *__restrict__ part) {
    const int F = L.F, H = L.H;
    const int64_t s0 = (int64_t)blockIdx.y * MLP_CHUNK, s1 = min(n, s0 + MLP_CHUNK);
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < L.count();
         p += (int64_t)gridDim.x * blockDim.x) {
        double g = 0.0;
        if (p < L.b1()) {                          // W1[j][i]: sum d1_j x_i
            const int j = (int)(p / F), i = (int)(p % F);
#pragma unroll 8
            for (int64_t s = s0; s < s1; s++) g += D1[s * H + j] * X[s * F + i];
        } else if (p < L.w2()) {                   // b1[j]
            const int j = (int)(p - L.b1());
#pragma unroll 8
            for (int64_t s = s0; s < s1; s++) g += D1[s * H + j];
        } else if (p < L.b2()) {                   // W2[k][j]: sum d2_k a1_j
            const int64_t q = p - L.w2();
            const int k = (int)(q / H), j = (int)(q % H);
#pragma unroll 8
            for (int64_t s = s0; s < s1; s++) g += D2[s * H + k] * A1[s * H + j];
        } else if (p < L.w3()) {                   // b2[k]
            const int k = (int)(p - L.b2());
#pragma unroll 8
            for (int64_t s = s0; s < s1; s++) g += D2[s * H + k];
        } else if (p < L.b3()) {                   // W3[k]: sum dy a2_k
            const int k = (int)(p - L.w3());
#pragma unroll 8
            for (int64_t s = s0; s < s1; s++) g += DY[s] * A2[s * H + k];
        } else {                                   // b3
            for (int64_t s = s0; s < s1; s++) g += DY[s];
        }
        part[(int64_t)blockIdx.y * L.count() + p] = g;
    }
}

__global__ void k_mlp_grad_sum(int nchunk, int64_t np, const double *__restrict__ part, double *__restrict__ G) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
        double g = 0.0;
        for (int c = 0; c < nchunk; c++) g += part[(int64_t)c * np + p];
        G[p] = g;
    }
}

__global__ void k_mlp_sqerr(int64_t n, const double *__restrict__ Y, const double *__restrict__ T,
                            double *__restrict__ out) {
    __shared__ double sh[256];
    double v = 0.0;
    for (int64_t s = threadIdx.x; s < n; s += blockDim.x) {
        const double d = Y[s] - T[s];
        v += d * d;
    }
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0] / (double)n;
}

// Adam (Kingma & Ba 2015), bias-corrected step sizes passed in
__global__ void k_mlp_adam(int64_t np, double *__restrict__ P, const double *__restrict__ G, double *__restrict__ M,
                           double *__restrict__ V, double lr, double b1, double b2, double eps, double bc1,
                           double bc2) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
        const double g = G[p];
        const double m = b1 * M[p] + (1.0 - b1) * g;
        const double v = b2 * V[p] + (1.0 - b2) * g * g;
        M[p] = m;
        V[p] = v;
        P[p] -= lr * (m / bc1) / (sqrt(v / bc2) + eps);
    }
}

template <typename T>
struct Buf {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t need(size_t cnt) {
        if (cnt <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, cnt * sizeof(T));
        if (e == cudaSuccess) n = cnt;
        return e;
    }
    ~Buf() {
        if (p) cudaFree(p);
    }
};

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(1024, (n + 127) / 128)); }

}  // namespace

struct pastix_gpu_mlp_s {
    int device = 0;
    Layout L{0, 0};
    cudaStream_t stream = nullptr;
    Buf<double> P, G, M, V, X, T, Y, A1, A2, DY, D2, D1, loss, part;
    int64_t step = 0;
};

#define MLP_CHECK(x)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) {                                                            \
            fprintf(stderr, "pastix_gpu_mlp: %s failed: %s\n", #x, cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? PASTIX_GPU_ERR_OUTOFMEMORY              \
                                                   : PASTIX_GPU_ERR_INTERNAL;               \
        }                                                                                   \
    } while (0)

extern "C" int pastix_gpu_mlp_init(pastix_gpu_mlp_t **pm, int device, int nfeat, int hidden, uint64_t seed) {
    if (!pm || nfeat <= 0 || nfeat > MLP_FMAX || hidden <= 0 || hidden > MLP_HMAX) return PASTIX_GPU_ERR_BADPARAMETER;
    *pm = nullptr;
    MLP_CHECK(cudaSetDevice(device));
    auto *m = new pastix_gpu_mlp_t();
    m->device = device;
    m->L = Layout{nfeat, hidden};
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete m;
        return PASTIX_GPU_ERR_INTERNAL;
    }
    const int64_t np = m->L.count();
    // He-uniform initialization of the weights, zero biases
    std::mt19937_64 rng(seed);
    std::vector<double> p(np, 0.0);
    auto fill = [&](int64_t off, int64_t cnt, int fan_in) {
        std::uniform_real_distribution<double> u(-std::sqrt(6.0 / fan_in), std::sqrt(6.0 / fan_in));
        for (int64_t i = 0; i < cnt; i++) p[off + i] = u(rng);
    };
    fill(m->L.w1(), (int64_t)hidden * nfeat, nfeat);
    fill(m->L.w2(), (int64_t)hidden * hidden, hidden);
    fill(m->L.w3(), hidden, hidden);
    if (m->P.need(np) || m->G.need(np) || m->M.need(np) || m->V.need(np) || m->loss.need(1)) {
        pastix_gpu_mlp_free(&m);
        return PASTIX_GPU_ERR_OUTOFMEMORY;
    }
    cudaMemcpy(m->P.p, p.data(), np * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemset(m->M.p, 0, np * sizeof(double));
    cudaMemset(m->V.p, 0, np * sizeof(double));
    *pm = m;
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_mlp_params(pastix_gpu_mlp_t *m, double *params, int64_t *count) {
    if (!m || !count) return PASTIX_GPU_ERR_BADPARAMETER;
    *count = m->L.count();
    if (params) {
        MLP_CHECK(cudaSetDevice(m->device));
        MLP_CHECK(cudaMemcpy(params, m->P.p, m->L.count() * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_mlp_set_params(pastix_gpu_mlp_t *m, const double *params) {
    if (!m || !params) return PASTIX_GPU_ERR_BADPARAMETER;
    MLP_CHECK(cudaSetDevice(m->device));
    MLP_CHECK(cudaMemcpy(m->P.p, params, m->L.count() * sizeof(double), cudaMemcpyHostToDevice));
    MLP_CHECK(cudaMemset(m->M.p, 0, m->L.count() * sizeof(double)));
    MLP_CHECK(cudaMemset(m->V.p, 0, m->L.count() * sizeof(double)));
    m->step = 0;
    return PASTIX_GPU_SUCCESS;
}

static int mlp_upload(pastix_gpu_mlp_t *m, int64_t n, const double *X, const double *T) {
    const int F = m->L.F, H = m->L.H;
    MLP_CHECK(m->X.need((size_t)n * F));
    MLP_CHECK(m->Y.need(n));
    MLP_CHECK(m->A1.need((size_t)n * H));
    MLP_CHECK(m->A2.need((size_t)n * H));
    MLP_CHECK(cudaMemcpyAsync(m->X.p, X, (size_t)n * F * sizeof(double), cudaMemcpyHostToDevice, m->stream));
    if (T) {
        MLP_CHECK(m->T.need(n));
        MLP_CHECK(m->DY.need(n));
        MLP_CHECK(m->D2.need((size_t)n * H));
        MLP_CHECK(m->D1.need((size_t)n * H));
        MLP_CHECK(m->part.need((size_t)((n + MLP_CHUNK - 1) / MLP_CHUNK) * m->L.count()));
        MLP_CHECK(cudaMemcpyAsync(m->T.p, T, n * sizeof(double), cudaMemcpyHostToDevice, m->stream));
    }
    return PASTIX_GPU_SUCCESS;
}

// forward + backward on the uploaded batch: G = dL/dP, loss written to m->loss
static void mlp_fwd_bwd(pastix_gpu_mlp_t *m, int64_t n) {
    const int g = grid_for(n);
    k_mlp_forward<<<g, 128, 0, m->stream>>>(n, m->L, m->X.p, m->P.p, m->A1.p, m->A2.p, m->Y.p);
    k_mlp_delta<<<g, 128, 0, m->stream>>>(n, m->L, m->P.p, m->A1.p, m->A2.p, m->Y.p, m->T.p, m->DY.p, m->D2.p,
                                         m->D1.p);
    const int nchunk = (int)((n + MLP_CHUNK - 1) / MLP_CHUNK);
    k_mlp_grad_partial<<<dim3((unsigned)((m->L.count() + 127) / 128), nchunk), 128, 0, m->stream>>>(
        n, m->L, m->X.p, m->A1.p, m->A2.p, m->DY.p, m->D2.p, m->D1.p, m->part.p);
    k_mlp_grad_sum<<<grid_for(m->L.count()), 128, 0, m->stream>>>(nchunk, m->L.count(), m->part.p, m->G.p);
    k_mlp_sqerr<<<1, 256, 0, m->stream>>>(n, m->Y.p, m->T.p, m->loss.p);
}

extern "C" int pastix_gpu_mlp_forward(pastix_gpu_mlp_t *m, int64_t n, const double *X, double *y) {
    if (!m || n <= 0 || !X || !y) return PASTIX_GPU_ERR_BADPARAMETER;
    MLP_CHECK(cudaSetDevice(m->device));
    int rc = mlp_upload(m, n, X, nullptr);
    if (rc) return rc;
    k_mlp_forward<<<grid_for(n), 128, 0, m->stream>>>(n, m->L, m->X.p, m->P.p, nullptr, nullptr, m->Y.p);
    MLP_CHECK(cudaGetLastError());
    MLP_CHECK(cudaMemcpyAsync(y, m->Y.p, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MLP_CHECK(cudaStreamSynchronize(m->stream));
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_mlp_gradient(pastix_gpu_mlp_t *m, int64_t n, const double *X, const double *t,
                                       double *grad, double *loss) {
    if (!m || n <= 0 || !X || !t) return PASTIX_GPU_ERR_BADPARAMETER;
    MLP_CHECK(cudaSetDevice(m->device));
    int rc = mlp_upload(m, n, X, t);
    if (rc) return rc;
    mlp_fwd_bwd(m, n);
    MLP_CHECK(cudaGetLastError());
    if (grad) MLP_CHECK(cudaMemcpyAsync(grad, m->G.p, m->L.count() * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    if (loss) MLP_CHECK(cudaMemcpyAsync(loss, m->loss.p, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MLP_CHECK(cudaStreamSynchronize(m->stream));
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_mlp_train(pastix_gpu_mlp_t *m, int64_t n, const double *X, const double *t, int steps,
                                    double lr, double *loss) {
    if (!m || n <= 0 || !X || !t || steps < 0 || !(lr > 0)) return PASTIX_GPU_ERR_BADPARAMETER;
    MLP_CHECK(cudaSetDevice(m->device));
    int rc = mlp_upload(m, n, X, t);
    if (rc) return rc;
    const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
    for (int it = 0; it < steps; it++) {
        mlp_fwd_bwd(m, n);
        m->step++;
        const double bc1 = 1.0 - std::pow(b1, (double)m->step), bc2 = 1.0 - std::pow(b2, (double)m->step);
        k_mlp_adam<<<grid_for(m->L.count()), 128, 0, m->stream>>>(m->L.count(), m->P.p, m->G.p, m->M.p, m->V.p, lr,
                                                                  b1, b2, eps, bc1, bc2);
    }
    // loss of the final parameters
    k_mlp_forward<<<grid_for(n), 128, 0, m->stream>>>(n, m->L, m->X.p, m->P.p, nullptr, nullptr, m->Y.p);
    k_mlp_sqerr<<<1, 256, 0, m->stream>>>(n, m->Y.p, m->T.p, m->loss.p);
    MLP_CHECK(cudaGetLastError());
    if (loss) MLP_CHECK(cudaMemcpyAsync(loss, m->loss.p, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MLP_CHECK(cudaStreamSynchronize(m->stream));
    return PASTIX_GPU_SUCCESS;
}

extern "C" void pastix_gpu_mlp_free(pastix_gpu_mlp_t **pm) {
    if (!pm || !*pm) return;
    pastix_gpu_mlp_t *m = *pm;
    cudaSetDevice(m->device);
    if (m->stream) {
        cudaStreamSynchronize(m->stream);
        cudaStreamDestroy(m->stream);
    }
    delete m;
    *pm = nullptr;
}
