// The expansion-order network: a 3 x 64 FP32 multilayer perceptron with
// hand-written forward, backward and Adam kernels. It maps a problem's features
// (k x box size per level, box and leaf-occupancy statistics of the tree, the
// requested tolerance) to the expansion order p and the depth offset. No
// counterpart in the reference, which takes p and the leaf size from the caller
// (HFMM.py:55-80); its choice is checked against the direct sum of
// test.py:11-18.
//
// Parameters, one flat FP32 array (row-major, input index first):
//   W1 [in][64], b1 [64], W2 [64][64], b2 [64], W3 [64][64], b3 [64],
//   W4 [64][out], b4 [out]
// Hidden activations tanh, linear output, loss = mean over samples and outputs
// of the squared error. One thread per sample runs the forward and backward
// recurrences against the weights staged in shared memory; each weight gradient
// is a sum over samples taken by one thread per parameter in FP64 (no atomics, so
// the gradient is deterministic); Adam updates one parameter per thread.
#include "hfmm_internal.cuh"

#include <cmath>
#include <vector>

namespace hfmm {

namespace {

constexpr int H = 64;
constexpr int MAX_IN = 64;
constexpr int MAX_OUT = 4;

struct Offs {
    int w1, b1, w2, b2, w3, b3, w4, b4, total;
};
__host__ __device__ inline Offs offsets(int in, int out) {
    Offs o;
    o.w1 = 0;
    o.b1 = o.w1 + in * H;
    o.w2 = o.b1 + H;
    o.b2 = o.w2 + H * H;
    o.w3 = o.b2 + H;
    o.b3 = o.w3 + H * H;
    o.w4 = o.b3 + H;
    o.b4 = o.w4 + H * out;
    o.total = o.b4 + out;
    return o;
}

// Per sample: the forward pass; with targets also the output gradient, the
// squared error and the deltas of the three hidden layers (tanh' = 1 - a^2).
__global__ void k_mlp_sample(const float* __restrict__ P, const float* __restrict__ X,
                             const float* __restrict__ T, int n, int in, int out, float* Y,
                             float* act, float* dlt, float* gout, float* sq) {
    extern __shared__ float w[];
    const Offs o = offsets(in, out);
    for (int i = threadIdx.x; i < o.total; i += blockDim.x) w[i] = P[i];
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float a1[H], a2[H], a3[H];
    const float* x = X + (int64_t)s * in;
    for (int j = 0; j < H; ++j) {
        float z = w[o.b1 + j];
        for (int i = 0; i < in; ++i) z = fmaf(x[i], w[o.w1 + i * H + j], z);
        a1[j] = tanhf(z);
    }
    for (int j = 0; j < H; ++j) {
        float z = w[o.b2 + j];
        for (int i = 0; i < H; ++i) z = fmaf(a1[i], w[o.w2 + i * H + j], z);
        a2[j] = tanhf(z);
    }
    for (int j = 0; j < H; ++j) {
        float z = w[o.b3 + j];
        for (int i = 0; i < H; ++i) z = fmaf(a2[i], w[o.w3 + i * H + j], z);
        a3[j] = tanhf(z);
    }
    float g[MAX_OUT];
    float e2 = 0.f;
    for (int c = 0; c < out; ++c) {
        float y = w[o.b4 + c];
        for (int i = 0; i < H; ++i) y = fmaf(a3[i], w[o.w4 + i * out + c], y);
        Y[(int64_t)s * out + c] = y;
        if (T) {
            const float e = y - T[(int64_t)s * out + c];
            e2 += e * e;
            g[c] = 2.0f * e / (float)((int64_t)n * out);
            gout[(int64_t)s * out + c] = g[c];
        }
    }
    if (!T) return;
    sq[s] = e2;
    float* A = act + (int64_t)s * 3 * H;
    float* D = dlt + (int64_t)s * 3 * H;
    float d3[H], d2[H];
    for (int j = 0; j < H; ++j) {
        float z = 0.f;
        for (int c = 0; c < out; ++c) z = fmaf(g[c], w[o.w4 + j * out + c], z);
        d3[j] = z * (1.0f - a3[j] * a3[j]);
    }
    for (int i = 0; i < H; ++i) {
        float z = 0.f;
        for (int j = 0; j < H; ++j) z = fmaf(w[o.w3 + i * H + j], d3[j], z);
        d2[i] = z * (1.0f - a2[i] * a2[i]);
    }
    for (int i = 0; i < H; ++i) {
        float z = 0.f;
        for (int j = 0; j < H; ++j) z = fmaf(w[o.w2 + i * H + j], d2[j], z);
        D[i] = z * (1.0f - a1[i] * a1[i]);
    }
    for (int j = 0; j < H; ++j) {
        A[j] = a1[j];
        A[H + j] = a2[j];
        A[2 * H + j] = a3[j];
        D[H + j] = d2[j];
        D[2 * H + j] = d3[j];
    }
}

// One thread per parameter: dL/dW[i][j] = sum_s in_s[i] * delta_s[j], dL/db[j] = sum_s delta_s[j].
__global__ void k_mlp_grad(const float* __restrict__ X, const float* __restrict__ act,
                           const float* __restrict__ dlt, const float* __restrict__ gout, int n,
                           int in, int out, float* G) {
    const Offs o = offsets(in, out);
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= o.total) return;
    const int64_t row = 3 * H;
    double acc = 0.0;
    if (p < o.b1) {
        const int i = p / H, j = p % H;
        for (int s = 0; s < n; ++s) acc += (double)X[(int64_t)s * in + i] * dlt[s * row + j];
    } else if (p < o.w2) {
        const int j = p - o.b1;
        for (int s = 0; s < n; ++s) acc += dlt[s * row + j];
    } else if (p < o.b2) {
        const int i = (p - o.w2) / H, j = (p - o.w2) % H;
        for (int s = 0; s < n; ++s) acc += (double)act[s * row + i] * dlt[s * row + H + j];
    } else if (p < o.w3) {
        const int j = p - o.b2;
        for (int s = 0; s < n; ++s) acc += dlt[s * row + H + j];
    } else if (p < o.b3) {
        const int i = (p - o.w3) / H, j = (p - o.w3) % H;
        for (int s = 0; s < n; ++s) acc += (double)act[s * row + H + i] * dlt[s * row + 2 * H + j];
    } else if (p < o.w4) {
        const int j = p - o.b3;
        for (int s = 0; s < n; ++s) acc += dlt[s * row + 2 * H + j];
    } else if (p < o.b4) {
        const int i = (p - o.w4) / out, c = (p - o.w4) % out;
        for (int s = 0; s < n; ++s) acc += (double)act[s * row + 2 * H + i] * gout[(int64_t)s * out + c];
    } else {
        const int c = p - o.b4;
        for (int s = 0; s < n; ++s) acc += gout[(int64_t)s * out + c];
    }
    G[p] = (float)acc;
}

// Adam (Kingma & Ba 2015, Algorithm 1) with bias corrections c1 = 1 - b1^t, c2 = 1 - b2^t.
__global__ void k_adam(float* P, const float* __restrict__ G, float* M, float* V, int np, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

struct Work {
    DevBuf<float> Y, act, dlt, gout, sq, G;
    Work(int n, int out, int np) {
        Y.alloc((size_t)n * out);
        act.alloc((size_t)n * 3 * H);
        dlt.alloc((size_t)n * 3 * H);
        gout.alloc((size_t)n * out);
        sq.alloc(n);
        G.alloc(np);
    }
};

void check_dims(int in, int out) {
    if (in < 1 || in > MAX_IN) throw Error{HFMM_ERR_ARG, "mlp: input width must be 1..64"};
    if (out < 1 || out > MAX_OUT) throw Error{HFMM_ERR_ARG, "mlp: output width must be 1..4"};
}

void sample_pass(const float* P, const float* X, const float* T, int n, int in, int out,
                 float* Y, Work* w, cudaStream_t s) {
    const Offs o = offsets(in, out);
    const int smem = o.total * (int)sizeof(float);
    HFMM_CUDA(cudaFuncSetAttribute(k_mlp_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    HFMM_LAUNCH(k_mlp_sample, (unsigned)ceil_div(n, 64), 64, (size_t)smem, s, P, X, T, n, in, out, Y,
                w ? w->act.p : nullptr, w ? w->dlt.p : nullptr, w ? w->gout.p : nullptr,
                w ? w->sq.p : nullptr);
}

double read_loss(Work& w, int n, int out, cudaStream_t s) {
    std::vector<float> sq(n);
    HFMM_CUDA(cudaMemcpyAsync(sq.data(), w.sq.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    HFMM_CUDA(cudaStreamSynchronize(s));
    double loss = 0.0;
    for (float v : sq) loss += v;
    return loss / ((double)n * out);
}

}  // namespace

int mlp_param_count(int in, int out) {
    check_dims(in, out);
    return offsets(in, out).total;
}

void mlp_forward(const float* P, const float* X, int n, int in, int out, float* Y, cudaStream_t s) {
    check_dims(in, out);
    sample_pass(P, X, nullptr, n, in, out, Y, nullptr, s);
}

double mlp_grad(const float* P, const float* X, const float* T, int n, int in, int out, float* G,
                cudaStream_t s) {
    check_dims(in, out);
    const int np = offsets(in, out).total;
    Work w(n, out, np);
    sample_pass(P, X, T, n, in, out, w.Y.p, &w, s);
    HFMM_LAUNCH(k_mlp_grad, (unsigned)ceil_div(np, 128), 128, 0, s, X, w.act.p, w.dlt.p, w.gout.p, n,
                in, out, G);
    return read_loss(w, n, out, s);
}

double mlp_train(float* P, float* adam_m, float* adam_v, int64_t t0, const float* X, const float* T,
                 int n, int in, int out, int steps, float lr, cudaStream_t s) {
    check_dims(in, out);
    const int np = offsets(in, out).total;
    Work w(n, out, np);
    const double b1 = 0.9, b2 = 0.999;
    for (int t = 1; t <= steps; ++t) {
        sample_pass(P, X, T, n, in, out, w.Y.p, &w, s);
        HFMM_LAUNCH(k_mlp_grad, (unsigned)ceil_div(np, 128), 128, 0, s, X, w.act.p, w.dlt.p, w.gout.p,
                    n, in, out, w.G.p);
        const double step = (double)(t0 + t);
        const float c1 = (float)(1.0 - std::pow(b1, step));
        const float c2 = (float)(1.0 - std::pow(b2, step));
        HFMM_LAUNCH(k_adam, (unsigned)ceil_div(np, 256), 256, 0, s, P, w.G.p, adam_m, adam_v, np, lr,
                    (float)b1, (float)b2, 1e-8f, c1, c2);
    }
    sample_pass(P, X, T, n, in, out, w.Y.p, &w, s);
    return read_loss(w, n, out, s);
}

}  // namespace hfmm

using namespace hfmm;

extern "C" {

int hfmm_mlp_param_count(int32_t in_dim, int32_t out_dim) {
    try {
        return mlp_param_count(in_dim, out_dim);
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

int hfmm_mlp_forward(const float* params, const float* X, int32_t n, int32_t in_dim,
                     int32_t out_dim, float* Y, void* stream) {
    if (!params || !X || !Y || n <= 0) return fail(HFMM_ERR_ARG, "invalid MLP arguments");
    try {
        require_device_ptr(params, "params");
        require_device_ptr(X, "X");
        require_device_ptr(Y, "Y");
        mlp_forward(params, X, n, in_dim, out_dim, Y, (cudaStream_t)stream);
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

int hfmm_mlp_grad(const float* params, const float* X, const float* T, int32_t n, int32_t in_dim,
                  int32_t out_dim, float* grad, double* loss, void* stream) {
    if (!params || !X || !T || !grad || n <= 0) return fail(HFMM_ERR_ARG, "invalid MLP arguments");
    try {
        require_device_ptr(params, "params");
        require_device_ptr(X, "X");
        require_device_ptr(T, "T");
        require_device_ptr(grad, "grad");
        const double l = mlp_grad(params, X, T, n, in_dim, out_dim, grad, (cudaStream_t)stream);
        if (loss) *loss = l;
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

int hfmm_mlp_train(float* params, float* adam_m, float* adam_v, int64_t step0, const float* X,
                   const float* T, int32_t n, int32_t in_dim, int32_t out_dim, int32_t steps,
                   float lr, double* loss, void* stream) {
    if (!params || !adam_m || !adam_v || !X || !T || n <= 0 || steps < 0 || step0 < 0)
        return fail(HFMM_ERR_ARG, "invalid MLP arguments");
    try {
        require_device_ptr(params, "params");
        require_device_ptr(adam_m, "adam_m");
        require_device_ptr(adam_v, "adam_v");
        require_device_ptr(X, "X");
        require_device_ptr(T, "T");
        const double l = mlp_train(params, adam_m, adam_v, step0, X, T, n, in_dim, out_dim, steps, lr,
                                   (cudaStream_t)stream);
        if (loss) *loss = l;
        return HFMM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.msg);
    }
}

}  // extern "C"
