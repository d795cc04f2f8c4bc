// dr_mlp.cu -- the learned parameter tuner: a 4-64-64-4 FP32 MLP with
// hand-written forward, backward and Adam kernels, and the proposal path that
// turns its outputs into engine parameters (with the endpoint-coverage check
// and the fallback to the reference heuristic).  No counterpart in the
// reference, which picks its parameters by fixed heuristics
// (mertens_dr.hpp:914-962, 1401-1419).
//
// Features (inputs):  log10 X, log2 HBM budget (bytes), SM count, batch size.
// Outputs:            cx, log2 fx, log2 u_cap, log2 segment length, where
//                     u = min(fx * (X / ln ln X)^(2/3), u_cap).
// Inputs and outputs are normalised by fixed affine maps (kIn*, kOut*) so the
// network works on O(1) values.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/dr_engine.h"
#include "dr_kernels.cuh"
#include "dr_params.hpp"

using namespace drb;

namespace {

constexpr int kIn = 4, kHid = 64, kOut = 4;
// parameter layout: W1[64][4] b1[64] W2[64][64] b2[64] W3[4][64] b3[4]
constexpr int oW1 = 0, oB1 = oW1 + kHid * kIn, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid,
              oB3 = oW3 + kOut * kHid, kParams = oB3 + kOut;  // 4740
constexpr int kMaxBatch = 4096;

// feature / target normalisation (shared with the numpy oracle in oracle/mlp_oracle.py)
constexpr float kInMean[kIn] = {13.0f, 35.0f, 148.0f, 0.0f};
constexpr float kInScale[kIn] = {3.0f, 3.0f, 64.0f, 8.0f};
constexpr float kOutMean[kOut] = {1.2f, 0.0f, 34.0f, 16.0f};
constexpr float kOutScale[kOut] = {0.5f, 1.5f, 4.0f, 1.5f};

// ---------------------------------------------------------------------------
// kernels: one 64-thread CTA per example
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64) mlp_forward_kernel(const float* __restrict__ P, const float* __restrict__ x,
                                                         int B, float* __restrict__ h1, float* __restrict__ h2,
                                                         float* __restrict__ y) {
    __shared__ float s_x[kIn], s_h1[kHid], s_h2[kHid];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    if (j < kIn) s_x[j] = x[b * kIn + j];
    __syncthreads();
    float a = P[oB1 + j];
#pragma unroll
    for (int i = 0; i < kIn; ++i) a = fmaf(P[oW1 + j * kIn + i], s_x[i], a);
    a = fmaxf(a, 0.f);
    s_h1[j] = a;
    if (h1) h1[b * kHid + j] = a;
    __syncthreads();
    float c = P[oB2 + j];
    for (int k = 0; k < kHid; ++k) c = fmaf(P[oW2 + j * kHid + k], s_h1[k], c);
    c = fmaxf(c, 0.f);
    s_h2[j] = c;
    if (h2) h2[b * kHid + j] = c;
    __syncthreads();
    if (j < kOut) {
        float o = P[oB3 + j];
        for (int k = 0; k < kHid; ++k) o = fmaf(P[oW3 + j * kHid + k], s_h2[k], o);
        y[b * kOut + j] = o;
    }
}

// Per-example gradient of L = mean over B*4 of (y - t)^2 into G[b][kParams];
// sq[b] = sum of squared errors of example b.
__global__ void __launch_bounds__(64) mlp_backward_kernel(const float* __restrict__ P, const float* __restrict__ x,
                                                          const float* __restrict__ t, const float* __restrict__ h1,
                                                          const float* __restrict__ h2, const float* __restrict__ y,
                                                          int B, float* __restrict__ G, float* __restrict__ sq) {
    __shared__ float s_x[kIn], s_h1[kHid], s_h2[kHid], s_dy[kOut], s_d2[kHid];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= B) return;
    float* g = G + (size_t)b * kParams;
    if (j < kIn) s_x[j] = x[b * kIn + j];
    s_h1[j] = h1[b * kHid + j];
    s_h2[j] = h2[b * kHid + j];
    if (j < kOut) {
        const float e = y[b * kOut + j] - t[b * kOut + j];
        s_dy[j] = 2.f * e / (float)(B * kOut);
    }
    __syncthreads();
    if (j == 0) {
        float s = 0.f;
        for (int o = 0; o < kOut; ++o) {
            const float e = y[b * kOut + o] - t[b * kOut + o];
            s += e * e;
        }
        sq[b] = s;
    }
    // layer 3: dW3[o][j] = dy[o] * h2[j], db3 = dy
#pragma unroll
    for (int o = 0; o < kOut; ++o) g[oW3 + o * kHid + j] = s_dy[o] * s_h2[j];
    if (j < kOut) g[oB3 + j] = s_dy[j];
    // dh2[j] = sum_o W3[o][j] dy[o], through the ReLU
    float d2 = 0.f;
#pragma unroll
    for (int o = 0; o < kOut; ++o) d2 = fmaf(P[oW3 + o * kHid + j], s_dy[o], d2);
    d2 = s_h2[j] > 0.f ? d2 : 0.f;
    s_d2[j] = d2;
    __syncthreads();
    // layer 2: dW2[j][k] = d2[j] * h1[k], db2 = d2
    for (int k = 0; k < kHid; ++k) g[oW2 + j * kHid + k] = d2 * s_h1[k];
    g[oB2 + j] = d2;
    // dh1[j] = sum_r W2[r][j] d2[r], through the ReLU
    float d1 = 0.f;
    for (int r = 0; r < kHid; ++r) d1 = fmaf(P[oW2 + r * kHid + j], s_d2[r], d1);
    d1 = s_h1[j] > 0.f ? d1 : 0.f;
#pragma unroll
    for (int i = 0; i < kIn; ++i) g[oW1 + j * kIn + i] = d1 * s_x[i];
    g[oB1 + j] = d1;
}

// grad[p] = sum_b G[b][p] in a fixed order (deterministic); loss = sum sq / (B*4)
__global__ void mlp_reduce_kernel(const float* __restrict__ G, const float* __restrict__ sq, int B,
                                  float* __restrict__ grad, float* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) {
        float s = 0.f;
        for (int b = 0; b < B; ++b) s += G[(size_t)b * kParams + p];
        grad[p] = s;
    }
    if (p == 0 && loss) {
        float s = 0.f;
        for (int b = 0; b < B; ++b) s += sq[b];
        *loss = s / (float)(B * kOut);
    }
}

// Adam (Kingma & Ba 2015) with bias correction.  The step count lives on the
// device (advanced by mlp_step_advance, a separate launch) so that one captured
// graph replays any number of steps.
__global__ void mlp_adam_kernel(float* __restrict__ P, const float* __restrict__ grad, float* __restrict__ m,
                                float* __restrict__ v, float* __restrict__ step, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const float t = *step + 1.f;
    if (p < kParams) {
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        const float g = grad[p];
        const float mm = b1 * m[p] + (1.f - b1) * g;
        const float vv = b2 * v[p] + (1.f - b2) * g * g;
        m[p] = mm;
        v[p] = vv;
        const float mh = mm / (1.f - powf(b1, t)), vh = vv / (1.f - powf(b2, t));
        P[p] -= lr * mh / (sqrtf(vh) + eps);
    }
}

__global__ void mlp_step_advance(float* step) { *step += 1.f; }

}  // namespace

struct dr_mlp {
    dr_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    float* P = nullptr;  // device parameters
    float* m = nullptr;
    float* v = nullptr;
    float* grad = nullptr;
    float* step = nullptr;
    float* loss = nullptr;
    float *x = nullptr, *t = nullptr, *h1 = nullptr, *h2 = nullptr, *y = nullptr, *G = nullptr, *sq = nullptr;
    int cap = 0;  // examples the work buffers hold
    cudaGraphExec_t train_graph = nullptr;
    int graph_B = 0;
    float graph_lr = 0.f;
};

namespace {

int mlp_fail(int code, const char* msg) { return record_error(code, msg); }

#define MCU(call)                                                 \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return mlp_fail(DR_ERR_CUDA, #call); \
    } while (0)

int mlp_reserve(dr_mlp* n, int B) {
    if (B <= n->cap) return DR_OK;
    if (n->train_graph) {
        cudaGraphExecDestroy(n->train_graph);
        n->train_graph = nullptr;
    }
    float** bufs[] = {&n->x, &n->t, &n->h1, &n->h2, &n->y, &n->G, &n->sq};
    for (float** b : bufs)
        if (*b) cudaFree(*b), *b = nullptr;
    const size_t sz[] = {(size_t)B * kIn, (size_t)B * kOut, (size_t)B * kHid, (size_t)B * kHid,
                         (size_t)B * kOut, (size_t)B * kParams, (size_t)B};
    for (int i = 0; i < 7; ++i) MCU(cudaMalloc(bufs[i], sz[i] * sizeof(float)));
    n->cap = B;
    return DR_OK;
}

// Training domain of the shipped network: X in [10^10, 10^16], budgets of
// 8..160 GiB.  Inputs outside it are clamped to its boundary: the outputs are
// already relative to the (X / ln ln X)^(2/3) law (fx, cx), so a proposal
// carried to a larger X keeps the scale-free part the network learned instead
// of extrapolating a ReLU network linearly.
constexpr double kLog10XMin = 10.0, kLog10XMax = 16.0, kLog2BudgetMin = 33.0, kLog2BudgetMax = 37.33;

void features(int64_t X, uint64_t budget, int sms, int batch, float out[kIn]) {
    const double lx = std::min(kLog10XMax, std::max(kLog10XMin, std::log10((double)std::max<int64_t>(X, 2))));
    const double lb = std::min(kLog2BudgetMax, std::max(kLog2BudgetMin, std::log2((double)std::max<uint64_t>(budget, 1))));
    const float raw[kIn] = {(float)lx, (float)lb, (float)sms, (float)std::log2((double)std::max(batch, 1))};
    for (int i = 0; i < kIn; ++i) out[i] = (raw[i] - kInMean[i]) / kInScale[i];
}

}  // namespace

// Host-side map from network outputs to engine parameters (exported for tests
// through dr_tuner_params).
static void outputs_to_params(int64_t X, const float yn[kOut], dr_params* p) {
    float o[kOut];
    for (int i = 0; i < kOut; ++i) o[i] = yn[i] * kOutScale[i] + kOutMean[i];
    const double cx = std::min(4.0, std::max(0.3, (double)o[0]));
    const double fx = std::exp2(std::min(4.0, std::max(-4.0, (double)o[1])));
    // the cap is an absolute size learned inside the training domain; for an X
    // outside it (whose features were clamped) it is carried along the same
    // X^(2/3) law as the rest of the proposal
    const double lx = std::log10((double)std::max<int64_t>(X, 2));
    const double lxc = std::min(kLog10XMax, std::max(kLog10XMin, lx));
    const double cap = std::exp2(std::min(41.0, std::max(20.0, (double)o[2]))) * std::pow(10.0, (2.0 / 3.0) * (lx - lxc));
    int seg = (int)std::lround(o[3]);
    seg = std::max(12, std::min(seg, 18));
    params_clear(p);
    const double loglogX = std::log(std::max(2.0, std::log((double)X)));
    int64_t u = (int64_t)std::min(cap, fx * std::pow((double)X / loglogX, 2.0 / 3.0));
    const int64_t S = isqrt_i64(X);
    const int64_t endpoint = (int64_t)(cx * std::sqrt((double)X)) + 1000;
    u = std::max(u, std::max(S + 1000, endpoint));
    u = ((u + 255) / 256) * 256;
    const int64_t e256 = (endpoint + 255) & ~255LL;
    p->u_total = u;
    // dense int16 tier as in the B200 policy: max(1.28e8, u/16) values, at most 4e9
    const int64_t dense_target = std::min<int64_t>(4000000000LL, std::max<int64_t>(128000000LL, u / 16));
    p->u_dense = std::min<int64_t>(u, std::max<int64_t>(e256, (dense_target + 255) & ~255LL));
    p->cx = cx;
    p->mu_limit = std::min(u, std::max(endpoint, X / u + 1000));
    p->segment_log2 = seg;
}

extern "C" {

int dr_mlp_create(dr_ctx* ctx, uint64_t seed, dr_mlp** out) {
    if (!out) return mlp_fail(DR_ERR_ARG, "out is NULL");
    *out = nullptr;
    dr_mlp* n = new dr_mlp();
    n->ctx = ctx;
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete n;
        return mlp_fail(DR_ERR_CUDA, "cudaStreamCreate failed");
    }
    float** bufs[] = {&n->P, &n->m, &n->v, &n->grad};
    for (float** b : bufs)
        if (cudaMalloc(b, kParams * sizeof(float)) != cudaSuccess) {
            dr_mlp_destroy(n);
            return mlp_fail(DR_ERR_NOMEM, "cudaMalloc failed");
        }
    if (cudaMalloc(&n->step, 2 * sizeof(float)) != cudaSuccess) {
        dr_mlp_destroy(n);
        return mlp_fail(DR_ERR_NOMEM, "cudaMalloc failed");
    }
    n->loss = n->step + 1;
    // He-uniform initialisation from a 64-bit LCG (host), biases zero
    std::vector<float> w(kParams, 0.f);
    uint64_t s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
    auto uni = [&]() {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        return (float)((double)(s >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    const float a1 = std::sqrt(6.f / kIn), a2 = std::sqrt(6.f / kHid), a3 = std::sqrt(6.f / kHid) * 0.1f;
    for (int i = 0; i < kHid * kIn; ++i) w[oW1 + i] = a1 * uni();
    for (int i = 0; i < kHid * kHid; ++i) w[oW2 + i] = a2 * uni();
    for (int i = 0; i < kOut * kHid; ++i) w[oW3 + i] = a3 * uni();
    int rc = dr_mlp_set_weights(n, w.data(), kParams);
    if (rc) {
        dr_mlp_destroy(n);
        return rc;
    }
    *out = n;
    return DR_OK;
}

int dr_mlp_destroy(dr_mlp* n) {
    if (!n) return DR_OK;
    if (n->train_graph) cudaGraphExecDestroy(n->train_graph);
    float* bufs[] = {n->P, n->m, n->v, n->grad, n->step, n->x, n->t, n->h1, n->h2, n->y, n->G, n->sq};
    for (float* b : bufs)
        if (b) cudaFree(b);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
    return DR_OK;
}

int64_t dr_mlp_num_params(void) { return kParams; }

int dr_mlp_set_weights(dr_mlp* n, const float* w, int64_t count) {
    if (!n || !w || count != kParams) return mlp_fail(DR_ERR_ARG, "dr_mlp_set_weights: need 4740 floats");
    MCU(cudaMemcpy(n->P, w, kParams * sizeof(float), cudaMemcpyHostToDevice));
    MCU(cudaMemset(n->m, 0, kParams * sizeof(float)));
    MCU(cudaMemset(n->v, 0, kParams * sizeof(float)));
    MCU(cudaMemset(n->step, 0, 2 * sizeof(float)));
    return DR_OK;
}

int dr_mlp_get_weights(dr_mlp* n, float* w, int64_t count) {
    if (!n || !w || count != kParams) return mlp_fail(DR_ERR_ARG, "dr_mlp_get_weights: need 4740 floats");
    MCU(cudaMemcpy(w, n->P, kParams * sizeof(float), cudaMemcpyDeviceToHost));
    return DR_OK;
}

// y = f(x) for B normalised feature rows (host arrays B x 4 -> B x 4).
int dr_mlp_forward(dr_mlp* n, const float* x, int64_t B, float* y) {
    if (!n || !x || !y || B < 1 || B > kMaxBatch) return mlp_fail(DR_ERR_ARG, "dr_mlp_forward: bad argument");
    int rc = mlp_reserve(n, (int)B);
    if (rc) return rc;
    MCU(cudaMemcpyAsync(n->x, x, B * kIn * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    mlp_forward_kernel<<<(unsigned)B, 64, 0, n->stream>>>(n->P, n->x, (int)B, nullptr, nullptr, n->y);
    MCU(cudaGetLastError());
    MCU(cudaMemcpyAsync(y, n->y, B * kOut * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    MCU(cudaStreamSynchronize(n->stream));
    return DR_OK;
}

// Gradient of the mean squared error over B examples (host arrays), no update.
int dr_mlp_grad(dr_mlp* n, const float* x, const float* t, int64_t B, float* grad, float* loss) {
    if (!n || !x || !t || !grad || B < 1 || B > kMaxBatch) return mlp_fail(DR_ERR_ARG, "dr_mlp_grad: bad argument");
    int rc = mlp_reserve(n, (int)B);
    if (rc) return rc;
    MCU(cudaMemcpyAsync(n->x, x, B * kIn * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    MCU(cudaMemcpyAsync(n->t, t, B * kOut * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    mlp_forward_kernel<<<(unsigned)B, 64, 0, n->stream>>>(n->P, n->x, (int)B, n->h1, n->h2, n->y);
    mlp_backward_kernel<<<(unsigned)B, 64, 0, n->stream>>>(n->P, n->x, n->t, n->h1, n->h2, n->y, (int)B, n->G, n->sq);
    mlp_reduce_kernel<<<(kParams + 255) / 256, 256, 0, n->stream>>>(n->G, n->sq, (int)B, n->grad, n->loss);
    MCU(cudaGetLastError());
    MCU(cudaMemcpyAsync(grad, n->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    float l = 0.f;
    MCU(cudaMemcpyAsync(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    MCU(cudaStreamSynchronize(n->stream));
    if (loss) *loss = l;
    return DR_OK;
}

// Full-batch Adam: `steps` updates on the B examples; each step is one replay
// of a captured graph (forward, backward, reduce, Adam, step counter).
int dr_mlp_train(dr_mlp* n, const float* x, const float* t, int64_t B, int steps, float lr, float* final_loss) {
    if (!n || !x || !t || B < 1 || B > kMaxBatch || steps < 0) return mlp_fail(DR_ERR_ARG, "dr_mlp_train: bad argument");
    int rc = mlp_reserve(n, (int)B);
    if (rc) return rc;
    MCU(cudaMemcpyAsync(n->x, x, B * kIn * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    MCU(cudaMemcpyAsync(n->t, t, B * kOut * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    if (!n->train_graph || n->graph_B != (int)B || n->graph_lr != lr) {
        if (n->train_graph) cudaGraphExecDestroy(n->train_graph);
        n->train_graph = nullptr;
        cudaGraph_t g = nullptr;
        MCU(cudaStreamBeginCapture(n->stream, cudaStreamCaptureModeThreadLocal));
        mlp_forward_kernel<<<(unsigned)B, 64, 0, n->stream>>>(n->P, n->x, (int)B, n->h1, n->h2, n->y);
        mlp_backward_kernel<<<(unsigned)B, 64, 0, n->stream>>>(n->P, n->x, n->t, n->h1, n->h2, n->y, (int)B, n->G,
                                                                n->sq);
        mlp_reduce_kernel<<<(kParams + 255) / 256, 256, 0, n->stream>>>(n->G, n->sq, (int)B, n->grad, n->loss);
        mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, n->stream>>>(n->P, n->grad, n->m, n->v, n->step, lr);
        mlp_step_advance<<<1, 1, 0, n->stream>>>(n->step);
        MCU(cudaStreamEndCapture(n->stream, &g));
        const cudaError_t e = cudaGraphInstantiate(&n->train_graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return mlp_fail(DR_ERR_CUDA, "training graph instantiation failed");
        n->graph_B = (int)B;
        n->graph_lr = lr;
    }
    for (int s = 0; s < steps; ++s) MCU(cudaGraphLaunch(n->train_graph, n->stream));
    float l = 0.f;
    MCU(cudaMemcpyAsync(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    MCU(cudaStreamSynchronize(n->stream));
    if (final_loss) *final_loss = l;
    return DR_OK;
}

// Engine parameters for X from the network's outputs (no check, no fallback).
int dr_tuner_params(int64_t X, const float* y_normalised, dr_params* out) {
    if (!y_normalised || !out || X < 1) return mlp_fail(DR_ERR_ARG, "dr_tuner_params: bad argument");
    outputs_to_params(X, y_normalised, out);
    return DR_OK;
}

// Normalised features of one query (the network's input row).
int dr_tuner_features(int64_t X, uint64_t hbm_budget, int sm_count, int batch, float* out4) {
    if (!out4) return mlp_fail(DR_ERR_ARG, "dr_tuner_features: out is NULL");
    features(X, hbm_budget, sm_count, batch, out4);
    return DR_OK;
}

// Shrink u (keeping cx, the dense tier and the endpoints) until the query's
// device footprint fits 90% of the budget: the budget is a hard constraint of
// the proposal, not a reason to discard it.
static void project_to_budget(int64_t X, uint64_t budget, dr_params* p) {
    if (!budget) return;
    for (int it = 0; it < 64 && dr_query_bytes(X, p) > budget / 10 * 9; ++it) {
        const int64_t S = isqrt_i64(X);
        const int64_t endpoint = (int64_t)(p->cx * std::sqrt((double)X)) + 1000;
        const int64_t floor_u = std::max(S + 1000, std::max(endpoint, p->u_dense));
        int64_t u = std::max(floor_u, (int64_t)((double)p->u_total * 0.9));
        u = ((u + 255) / 256) * 256;
        if (u >= p->u_total) break;
        p->u_total = u;
        p->mu_limit = std::min(u, std::max(endpoint, X / u + 1000));
    }
}

// The learned tuner's proposal for X: network inference on the device, mapped
// to parameters and projected onto the device budget, then the endpoint-
// coverage check; a proposal that fails it is replaced by the reference's
// default heuristic (*fallback = 1).
int dr_tuner_propose(dr_mlp* n, int64_t X, uint64_t hbm_budget, int sm_count, int batch, dr_params* out,
                     int* fallback) {
    if (!n || !out) return mlp_fail(DR_ERR_ARG, "dr_tuner_propose: bad argument");
    float f[kIn], y[kOut];
    features(X, hbm_budget, sm_count, batch, f);
    int rc = dr_mlp_forward(n, f, 1, y);
    if (rc) return rc;
    outputs_to_params(X, y, out);
    if (X > 0) project_to_budget(X, hbm_budget, out);
    int fb = 0;
    if (X < 1 || dr_check_params(X, out, hbm_budget) != DR_OK) {
        fb = 1;
        rc = dr_default_params(X, DR_POLICY_REFERENCE, out);
        if (rc) return rc;
    }
    if (fallback) *fallback = fb;
    return DR_OK;
}

}  // extern "C"
