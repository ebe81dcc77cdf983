// up_costmodel.cu — the learned cost model (ultraprecise_costmodel.h): a
// UP_CM_FEATURES -> 64 -> 64 -> 1 perceptron with SiLU activations that
// predicts log(ms) of an expression launch, trained on the GPU by the kernels
// below.
//
// The network is tiny (5313 parameters) and its data set is a few hundred
// measured launches, so every kernel keeps the whole parameter vector in
// shared memory.  Training runs one kernel per step in one CTA: gather the
// step's mini-batch (<= 128 samples) by index, forward pass one thread per
// sample, backward pass one thread per sample (per-sample deltas), then
// weight gradients one thread per parameter (sums over the batch from shared
// memory) followed by the Adam update of that parameter — no atomics, no
// second launch.  Prediction is a grid of CTAs, one thread per sample.  The
// arithmetic is fp32 SIMT: the shapes are far below what tensor-core tiles
// pay off on, and a step is bound by launch latency, not by flops.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/ultraprecise_costmodel.h"
#include "up_internal.h"

namespace upi {
namespace {

constexpr int F = UP_CM_FEATURES;
constexpr int H = UP_CM_HIDDEN;
constexpr int NP = UP_CM_PARAMS;
constexpr int BMAX = UP_CM_BATCH_MAX;
constexpr int oW1 = 0;
constexpr int oB1 = oW1 + F * H;
constexpr int oW2 = oB1 + H;
constexpr int oB2 = oW2 + H * H;
constexpr int oW3 = oB2 + H;
constexpr int oB3 = oW3 + H;
static_assert(oB3 + 1 == NP, "parameter layout");
constexpr int HS = H + 1;  // padded row stride of the per-sample activations (no bank conflicts)
constexpr int kStepThreads = 256;

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigmoid(z);
    return s * (1.0f + z * (1.0f - s));
}

// Dynamic shared memory of the step kernel, in floats.
constexpr int kStepSmemFloats = NP + BMAX * F + 4 * BMAX * HS + 2 * BMAX + 32;

// One training step (or, with adam == 0, gradients only) over the samples
// idx[0..n) of X (rows of F floats) and Y.
__global__ void __launch_bounds__(kStepThreads) k_mlp_step(float* __restrict__ params, float* __restrict__ adam_m,
                                                           float* __restrict__ adam_v,
                                                           float* __restrict__ grads_out,
                                                           const float* __restrict__ X, const float* __restrict__ Y,
                                                           const int* __restrict__ idx, int n, int adam, float lr,
                                                           float bc1, float bc2, float* __restrict__ loss_out) {
    extern __shared__ float sm[];
    float* P = sm;                     // parameters
    float* Xs = P + NP;                // [BMAX][F]
    float* Z1 = Xs + BMAX * F;         // [BMAX][HS]: pre-activations of layer 1, then their deltas
    float* A1 = Z1 + BMAX * HS;        // activations of layer 1
    float* Z2 = A1 + BMAX * HS;        // pre-activations of layer 2, then their deltas
    float* A2 = Z2 + BMAX * HS;        // activations of layer 2
    float* DO = A2 + BMAX * HS;        // [BMAX]: d loss / d output
    float* Ys = DO + BMAX;             // [BMAX]
    float* red = Ys + BMAX;            // [32]: loss reduction
    const int tid = threadIdx.x;
    for (int i = tid; i < NP; i += blockDim.x) P[i] = params[i];
    for (int i = tid; i < n * F; i += blockDim.x) Xs[i] = X[(size_t)idx[i / F] * F + (i % F)];
    for (int i = tid; i < n; i += blockDim.x) Ys[i] = Y[idx[i]];
    if (tid < 32) red[tid] = 0.0f;
    __syncthreads();
    // forward, one thread per sample
    float se = 0.0f;
    if (tid < n) {
        const float* x = Xs + tid * F;
        float* z1 = Z1 + tid * HS;
        float* a1 = A1 + tid * HS;
        for (int h = 0; h < H; h++) {
            float z = P[oB1 + h];
#pragma unroll
            for (int f = 0; f < F; f++) z = fmaf(x[f], P[oW1 + f * H + h], z);
            z1[h] = z;
            a1[h] = silu(z);
        }
        float* z2 = Z2 + tid * HS;
        float* a2 = A2 + tid * HS;
        float out = P[oB3];
        for (int j = 0; j < H; j++) {
            float z = P[oB2 + j];
            for (int i = 0; i < H; i++) z = fmaf(a1[i], P[oW2 + i * H + j], z);
            z2[j] = z;
            const float a = silu(z);
            a2[j] = a;
            out = fmaf(a, P[oW3 + j], out);
        }
        const float e = out - Ys[tid];
        se = e * e;
        DO[tid] = 2.0f * e / (float)n;  // d(mean squared error)/d out
    }
    // backward, one thread per sample: deltas of layer 2, then of layer 1
    if (tid < n) {
        float* z2 = Z2 + tid * HS;
        float* z1 = Z1 + tid * HS;
        const float d = DO[tid];
        for (int j = 0; j < H; j++) z2[j] = P[oW3 + j] * d * dsilu(z2[j]);  // now dL/dz2
        for (int i = 0; i < H; i++) {
            float g = 0.0f;
            for (int j = 0; j < H; j++) g = fmaf(P[oW2 + i * H + j], z2[j], g);
            z1[i] = g * dsilu(z1[i]);  // now dL/dz1
        }
    }
    // loss: warp sums, then one atomic per warp into shared memory
    for (int o = 16; o > 0; o >>= 1) se += __shfl_down_sync(0xffffffffu, se, o);
    if ((tid & 31) == 0) atomicAdd(&red[0], se);
    __syncthreads();
    // weight gradients, one thread per parameter, then the update
    for (int p = tid; p < NP; p += blockDim.x) {
        float g = 0.0f;
        if (p < oB1) {
            const int f = p / H, h = p % H;
            for (int s = 0; s < n; s++) g = fmaf(Xs[s * F + f], Z1[s * HS + h], g);
        } else if (p < oW2) {
            const int h = p - oB1;
            for (int s = 0; s < n; s++) g += Z1[s * HS + h];
        } else if (p < oB2) {
            const int i = (p - oW2) / H, j = (p - oW2) % H;
            for (int s = 0; s < n; s++) g = fmaf(A1[s * HS + i], Z2[s * HS + j], g);
        } else if (p < oW3) {
            const int j = p - oB2;
            for (int s = 0; s < n; s++) g += Z2[s * HS + j];
        } else if (p < oB3) {
            const int j = p - oW3;
            for (int s = 0; s < n; s++) g = fmaf(A2[s * HS + j], DO[s], g);
        } else {
            for (int s = 0; s < n; s++) g += DO[s];
        }
        if (grads_out) grads_out[p] = g;
        if (adam) {
            // Adam (Kingma & Ba 2015): beta1 0.9, beta2 0.999, eps 1e-8;
            // bc1, bc2 = 1 / (1 - beta^t) for this step t
            const float m = 0.9f * adam_m[p] + 0.1f * g;
            const float v = 0.999f * adam_v[p] + 0.001f * g * g;
            adam_m[p] = m;
            adam_v[p] = v;
            params[p] = P[p] - lr * (m * bc1) / (sqrtf(v * bc2) + 1e-8f);
        }
    }
    if (tid == 0 && loss_out) *loss_out = red[0] / (float)(n > 0 ? n : 1);
}

// Predictions: one thread per sample, parameters in shared memory.
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ params, const float* __restrict__ X,
                                                     int n, float* __restrict__ out) {
    __shared__ float P[NP];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[F];
#pragma unroll
    for (int f = 0; f < F; f++) x[f] = X[(size_t)s * F + f];
    float a1[H];
#pragma unroll 4
    for (int h = 0; h < H; h++) {
        float z = P[oB1 + h];
#pragma unroll
        for (int f = 0; f < F; f++) z = fmaf(x[f], P[oW1 + f * H + h], z);
        a1[h] = silu(z);
    }
    float o = P[oB3];
    for (int j = 0; j < H; j++) {
        float z = P[oB2 + j];
#pragma unroll
        for (int i = 0; i < H; i++) z = fmaf(a1[i], P[oW2 + i * H + j], z);
        o = fmaf(silu(z), P[oW3 + j], o);
    }
    out[s] = o;
}

}  // namespace
}  // namespace upi

using namespace upi;

struct up_costmodel {
    std::mutex mu;
    std::vector<float> params;      // host copy, kept current
    float norm[2 * UP_CM_FEATURES + 2];  // feature means, feature stds, target mean, target std
    int device = -1;
    float* d_params = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_loss = nullptr;
    cudaStream_t stream = nullptr;
    // further trained networks whose predictions are averaged with this one's
    struct Member {
        std::vector<float> params;
        float norm[2 * UP_CM_FEATURES + 2];
        float* d_params = nullptr;
    };
    std::vector<Member> members;
    float guard = 0.0f;  // choose_tpv keeps the width rule unless this fraction of time is predicted saved
    ~up_costmodel() {
        if (stream) cudaStreamSynchronize(stream);
        for (float* p : {d_params, d_m, d_v, d_loss})
            if (p) cudaFree(p);
        for (auto& mb : members)
            if (mb.d_params) cudaFree(mb.d_params);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

up_status cm_cuda(cudaError_t e, const char* what) {
    cudaGetLastError();
    return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define CM_CUDA(call)                                  \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cm_cuda(e_, #call); \
    } while (0)

// Device buffers and the private stream, created on first use on the current
// device; the host parameters are uploaded.
up_status cm_ready(up_costmodel* m) {
    int dev = -1;
    CM_CUDA(cudaGetDevice(&dev));
    if (m->d_params && m->device == dev) return UP_OK;
    if (m->d_params) return fail(UP_ERR_UNSUPPORTED, "cost model used on a second device");
    CM_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    CM_CUDA(cudaMalloc(&m->d_params, NP * sizeof(float)));
    CM_CUDA(cudaMalloc(&m->d_m, NP * sizeof(float)));
    CM_CUDA(cudaMalloc(&m->d_v, NP * sizeof(float)));
    CM_CUDA(cudaMalloc(&m->d_loss, sizeof(float)));
    CM_CUDA(cudaMemcpyAsync(m->d_params, m->params.data(), NP * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    CM_CUDA(cudaStreamSynchronize(m->stream));
    CM_CUDA(cudaFuncSetAttribute((const void*)k_mlp_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kStepSmemFloats * sizeof(float))));
    m->device = dev;
    return UP_OK;
}

// A device buffer that frees itself.
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

void standardise(const float* x, int n, const float* norm, float* out) {
    for (int i = 0; i < n; i++)
        for (int f = 0; f < F; f++) out[(size_t)i * F + f] = (x[(size_t)i * F + f] - norm[f]) / norm[F + f];
}

// One network's prediction (log ms) with its own parameters and standardisation.
up_status predict_one(up_costmodel* m, const float* d_params, const float* norm, const float* feats, int n,
                      float* log_ms) {
    std::vector<float> xs((size_t)n * F);
    standardise(feats, n, norm, xs.data());
    DevBuf dx, dout;
    CM_CUDA(cudaMalloc(&dx.p, xs.size() * sizeof(float)));
    CM_CUDA(cudaMalloc(&dout.p, (size_t)n * sizeof(float)));
    CM_CUDA(cudaMemcpyAsync(dx.p, xs.data(), xs.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    k_mlp_forward<<<(unsigned)((n + 127) / 128), 128, 0, m->stream>>>(d_params, (const float*)dx.p, n,
                                                                       (float*)dout.p);
    CM_CUDA(cudaGetLastError());
    std::vector<float> o(n);
    CM_CUDA(cudaMemcpyAsync(o.data(), dout.p, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    CM_CUDA(cudaStreamSynchronize(m->stream));
    for (int i = 0; i < n; i++) log_ms[i] = o[i] * norm[2 * F + 1] + norm[2 * F];
    return UP_OK;
}

// The model's prediction: the mean log ms of its network and its members.
up_status predict_locked(up_costmodel* m, const float* feats, int n, float* log_ms) {
    up_status st = cm_ready(m);
    if (st != UP_OK) return st;
    if ((st = predict_one(m, m->d_params, m->norm, feats, n, log_ms)) != UP_OK) return st;
    if (m->members.empty()) return UP_OK;
    std::vector<double> sum(log_ms, log_ms + n);
    std::vector<float> one(n);
    for (auto& mb : m->members) {
        if (!mb.d_params) {
            CM_CUDA(cudaMalloc(&mb.d_params, NP * sizeof(float)));
            CM_CUDA(cudaMemcpyAsync(mb.d_params, mb.params.data(), NP * sizeof(float), cudaMemcpyHostToDevice,
                                    m->stream));
        }
        if ((st = predict_one(m, mb.d_params, mb.norm, feats, n, one.data())) != UP_OK) return st;
        for (int i = 0; i < n; i++) sum[i] += one[i];
    }
    for (int i = 0; i < n; i++) log_ms[i] = (float)(sum[i] / (double)(m->members.size() + 1));
    return UP_OK;
}

std::mutex g_default_mu;
up_costmodel* g_default = nullptr;

}  // namespace

namespace upi {
CostChoice default_model_choose_tpv(const up_expr_node* nodes, int n_nodes, int root, const up_col_type* cols,
                                    int n_cols) {
    CostChoice c;
    std::lock_guard<std::mutex> g(g_default_mu);
    if (!g_default) return c;
    int32_t tpv = 1;
    if (up_costmodel_choose_tpv(g_default, nodes, n_nodes, root, cols, n_cols, UP_CM_ROWS_HINT, &tpv, nullptr) ==
        UP_OK) {
        c.valid = true;
        c.tpv = tpv;
    }
    return c;
}
}  // namespace upi

extern "C" {

up_status up_costmodel_create(uint64_t seed, up_costmodel** out) {
    if (!out) return fail(UP_ERR_INVALID_ARG, "out is NULL");
    up_costmodel* m = new up_costmodel();
    m->params.assign(NP, 0.0f);
    std::mt19937_64 rng(seed);
    auto init = [&](int off, int fan_in, int count) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)fan_in));
        for (int i = 0; i < count; i++) m->params[off + i] = nd(rng);
    };
    init(oW1, F, F * H);
    init(oW2, H, H * H);
    init(oW3, H, H);
    for (int f = 0; f < F; f++) {
        m->norm[f] = 0.0f;
        m->norm[F + f] = 1.0f;
    }
    m->norm[2 * F] = 0.0f;
    m->norm[2 * F + 1] = 1.0f;
    *out = m;
    return UP_OK;
}

void up_costmodel_release(up_costmodel* m) {
    if (!m) return;
    {
        std::lock_guard<std::mutex> g(g_default_mu);
        if (g_default == m) g_default = nullptr;
    }
    delete m;
}

up_status up_costmodel_expr_features(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                                     const up_col_type* cols, int32_t n_cols, int32_t threads_per_value,
                                     int64_t rows, float* features, int32_t* coop_ok) {
    if (!nodes || n_nodes <= 0 || !features) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    if (threads_per_value != 1 && threads_per_value != 2 && threads_per_value != 4 && threads_per_value != 8 &&
        threads_per_value != 16 && threads_per_value != 32)
        return fail(UP_ERR_INVALID_ARG, "threads_per_value must be 1, 2, 4, 8, 16 or 32");
    bool ok = false;
    up_status st = expr_cost_features(nodes, n_nodes, root, cols, n_cols, threads_per_value, rows, features, &ok);
    if (coop_ok) *coop_ok = ok ? 1 : 0;
    return st;
}

up_status up_costmodel_train(up_costmodel* m, const float* features, const float* targets, int32_t n,
                             int32_t epochs, int32_t batch, float lr, uint64_t seed, float* final_loss) {
    if (!m || !features || !targets || n <= 0) return fail(UP_ERR_INVALID_ARG, "bad training set");
    if (batch <= 0 || batch > BMAX || epochs <= 0 || !(lr > 0.0f)) return fail(UP_ERR_INVALID_ARG, "bad schedule");
    std::lock_guard<std::mutex> g(m->mu);
    up_status st = cm_ready(m);
    if (st != UP_OK) return st;
    // standardisation statistics of this training set
    for (int f = 0; f < F; f++) {
        double s = 0, s2 = 0;
        for (int i = 0; i < n; i++) {
            const double v = features[(size_t)i * F + f];
            s += v;
            s2 += v * v;
        }
        const double mean = s / n, var = std::max(0.0, s2 / n - mean * mean);
        m->norm[f] = (float)mean;
        m->norm[F + f] = (float)std::max(std::sqrt(var), 1e-3);
    }
    {
        double s = 0, s2 = 0;
        for (int i = 0; i < n; i++) {
            s += targets[i];
            s2 += (double)targets[i] * targets[i];
        }
        const double mean = s / n, var = std::max(0.0, s2 / n - mean * mean);
        m->norm[2 * F] = (float)mean;
        m->norm[2 * F + 1] = (float)std::max(std::sqrt(var), 1e-3);
    }
    std::vector<float> xs((size_t)n * F), ys(n);
    standardise(features, n, m->norm, xs.data());
    for (int i = 0; i < n; i++) ys[i] = (targets[i] - m->norm[2 * F]) / m->norm[2 * F + 1];
    // every epoch's shuffled order, uploaded once
    std::vector<int> order((size_t)epochs * n);
    std::mt19937_64 rng(seed);
    for (int e = 0; e < epochs; e++) {
        int* o = order.data() + (size_t)e * n;
        for (int i = 0; i < n; i++) o[i] = i;
        std::shuffle(o, o + n, rng);
    }
    DevBuf dx, dy, didx;
    CM_CUDA(cudaMalloc(&dx.p, xs.size() * sizeof(float)));
    CM_CUDA(cudaMalloc(&dy.p, ys.size() * sizeof(float)));
    CM_CUDA(cudaMalloc(&didx.p, order.size() * sizeof(int)));
    cudaStream_t s = m->stream;
    CM_CUDA(cudaMemcpyAsync(dx.p, xs.data(), xs.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    CM_CUDA(cudaMemcpyAsync(dy.p, ys.data(), ys.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    CM_CUDA(cudaMemcpyAsync(didx.p, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CM_CUDA(cudaMemsetAsync(m->d_m, 0, NP * sizeof(float), s));
    CM_CUDA(cudaMemsetAsync(m->d_v, 0, NP * sizeof(float), s));
    const size_t smem = kStepSmemFloats * sizeof(float);
    int t = 0;
    for (int e = 0; e < epochs; e++)
        for (int b = 0; b < n; b += batch) {
            const int nb = std::min(batch, n - b);
            t++;
            const float bc1 = (float)(1.0 / (1.0 - std::pow(0.9, t)));
            const float bc2 = (float)(1.0 / (1.0 - std::pow(0.999, t)));
            k_mlp_step<<<1, kStepThreads, smem, s>>>(m->d_params, m->d_m, m->d_v, nullptr, (const float*)dx.p,
                                                    (const float*)dy.p, (const int*)didx.p + (size_t)e * n + b, nb, 1,
                                                    lr, bc1, bc2, nullptr);
        }
    CM_CUDA(cudaGetLastError());
    CM_CUDA(cudaMemcpyAsync(m->params.data(), m->d_params, NP * sizeof(float), cudaMemcpyDeviceToHost, s));
    CM_CUDA(cudaStreamSynchronize(s));
    if (final_loss) {
        std::vector<float> pred(n);
        // predictions in standardised units: undo the target scaling of predict
        std::vector<float> raw(features, features + (size_t)n * F);
        st = predict_locked(m, raw.data(), n, pred.data());
        if (st != UP_OK) return st;
        double se = 0;
        for (int i = 0; i < n; i++) {
            const double e = (pred[i] - targets[i]) / m->norm[2 * F + 1];
            se += e * e;
        }
        *final_loss = (float)(se / n);
    }
    return UP_OK;
}

up_status up_costmodel_predict(up_costmodel* m, const float* features, int32_t n, float* log_ms) {
    if (!m || !features || !log_ms || n < 0) return fail(UP_ERR_INVALID_ARG, "bad arguments");
    if (n == 0) return UP_OK;
    std::lock_guard<std::mutex> g(m->mu);
    return predict_locked(m, features, n, log_ms);
}

up_status up_costmodel_gradients(up_costmodel* m, const float* features, const float* targets, int32_t n,
                                 float* grads, float* loss) {
    if (!m || !features || !targets || !grads || n <= 0 || n > BMAX) return fail(UP_ERR_INVALID_ARG, "bad batch");
    std::lock_guard<std::mutex> g(m->mu);
    up_status st = cm_ready(m);
    if (st != UP_OK) return st;
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    DevBuf dx, dy, di, dg;
    CM_CUDA(cudaMalloc(&dx.p, (size_t)n * F * sizeof(float)));
    CM_CUDA(cudaMalloc(&dy.p, (size_t)n * sizeof(float)));
    CM_CUDA(cudaMalloc(&di.p, (size_t)n * sizeof(int)));
    CM_CUDA(cudaMalloc(&dg.p, NP * sizeof(float)));
    cudaStream_t s = m->stream;
    CM_CUDA(cudaMemcpyAsync(dx.p, features, (size_t)n * F * sizeof(float), cudaMemcpyHostToDevice, s));
    CM_CUDA(cudaMemcpyAsync(dy.p, targets, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s));
    CM_CUDA(cudaMemcpyAsync(di.p, idx.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
    k_mlp_step<<<1, kStepThreads, kStepSmemFloats * sizeof(float), s>>>(
        m->d_params, m->d_m, m->d_v, (float*)dg.p, (const float*)dx.p, (const float*)dy.p, (const int*)di.p, n, 0,
        0.0f, 1.0f, 1.0f, m->d_loss);
    CM_CUDA(cudaGetLastError());
    float l = 0.0f;
    CM_CUDA(cudaMemcpyAsync(grads, dg.p, NP * sizeof(float), cudaMemcpyDeviceToHost, s));
    CM_CUDA(cudaMemcpyAsync(&l, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    CM_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = l;
    return UP_OK;
}

up_status up_costmodel_get_params(const up_costmodel* m, float* params, float* norm) {
    if (!m || !params) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    std::memcpy(params, m->params.data(), NP * sizeof(float));
    if (norm) std::memcpy(norm, m->norm, sizeof m->norm);
    return UP_OK;
}

up_status up_costmodel_set_params(up_costmodel* m, const float* params, const float* norm) {
    if (!m || !params) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    std::lock_guard<std::mutex> g(m->mu);
    std::memcpy(m->params.data(), params, NP * sizeof(float));
    if (norm) std::memcpy(m->norm, norm, sizeof m->norm);
    if (m->d_params) {
        CM_CUDA(cudaMemcpyAsync(m->d_params, m->params.data(), NP * sizeof(float), cudaMemcpyHostToDevice, m->stream));
        CM_CUDA(cudaStreamSynchronize(m->stream));
    }
    return UP_OK;
}

up_status up_costmodel_choose_tpv(up_costmodel* m, const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                                  const up_col_type* cols, int32_t n_cols, int64_t rows, int32_t* tpv,
                                  float* pred_ms) {
    if (!m || !tpv) return fail(UP_ERR_INVALID_ARG, "NULL arguments");
    static const int cand[6] = {1, 2, 4, 8, 16, 32};
    float feats[6 * F];
    int32_t coop = 0;
    up_status st = up_costmodel_expr_features(nodes, n_nodes, root, cols, n_cols, 1, rows, feats, &coop);
    if (st != UP_OK) return st;
    int nc = 1;
    if (coop)
        for (; nc < 6; nc++) {
            st = up_costmodel_expr_features(nodes, n_nodes, root, cols, n_cols, cand[nc], rows, feats + nc * F,
                                            nullptr);
            if (st != UP_OK) return st;
        }
    float pred[6];
    {
        std::lock_guard<std::mutex> g(m->mu);
        st = predict_locked(m, feats, nc, pred);
    }
    if (st != UP_OK) return st;
    int best = 0;
    for (int i = 1; i < nc; i++)
        if (pred[i] < pred[best]) best = i;
    if (m->guard > 0.0f && nc > 1) {
        // keep the width rule's choice unless the model predicts it saves at least `guard` of the time
        std::vector<NodeFacts> f;
        std::vector<int> topo;
        if (analyze_nodes(nodes, n_nodes, cols, n_cols, f, topo, {root}) == UP_OK) {
            const int rt = rule_threads_per_value(nodes, f, topo);
            for (int i = 0; i < nc; i++)
                if (cand[i] == rt && pred[best] > pred[i] + std::log(1.0f - m->guard)) best = i;
        }
    }
    *tpv = cand[best];
    if (pred_ms) *pred_ms = std::exp(pred[best]);
    return UP_OK;
}

up_status up_costmodel_add_member(up_costmodel* m, const up_costmodel* other) {
    if (!m || !other || m == other) return fail(UP_ERR_INVALID_ARG, "bad models");
    std::lock_guard<std::mutex> g(m->mu);
    up_costmodel::Member mb;
    mb.params = other->params;
    std::memcpy(mb.norm, other->norm, sizeof mb.norm);
    m->members.push_back(std::move(mb));
    return UP_OK;
}

up_status up_costmodel_set_guard(up_costmodel* m, float margin) {
    if (!m || !(margin >= 0.0f) || !(margin < 1.0f)) return fail(UP_ERR_INVALID_ARG, "guard must be in [0, 1)");
    std::lock_guard<std::mutex> g(m->mu);
    m->guard = margin;
    return UP_OK;
}

up_status up_costmodel_set_default(up_costmodel* m) {
    std::lock_guard<std::mutex> g(g_default_mu);
    g_default = m;
    return UP_OK;
}

}  // extern "C"
