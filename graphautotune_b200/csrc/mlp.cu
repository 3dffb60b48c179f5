// The learned cost model's network: a 3-layer FP32 perceptron
//   h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), y = h2 w3 + b3
// with hand-written forward, backward (mean squared error) and Adam kernels.
// It replaces the reference tuner's XGBoost regressor
// (tuning/tuning/role/modeling.py:16-162): it maps (schedule, configuration,
// graph statistics) features to log run time and ranks candidate
// configurations; it is trained on the GPU from timings the engine itself
// records.
//
// Sizes are tiny (input <= 64 features, hidden = 64), so the kernels are
// plain CUDA-core FP32: one warp per sample row for the forward pass and the
// per-row deltas (weights staged in shared memory), then one thread per
// parameter summing its gradient over the rows in order (deterministic, no
// atomics).  Tensor cores would not pay at this size.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/gat.h"

namespace {

constexpr int kHidden = 64;
constexpr int kMaxIn = 64;
constexpr int kRowsPerCta = 8;  // one warp per row, 256 threads

thread_local std::string g_mlp_err;

struct Shape {
    int in;
    // parameter offsets in the flat vector
    int w1, b1, w2, b2, w3, b3, total;
    explicit Shape(int in_) : in(in_) {
        w1 = 0;
        b1 = w1 + in * kHidden;
        w2 = b1 + kHidden;
        b2 = w2 + kHidden * kHidden;
        w3 = b2 + kHidden;
        b3 = w3 + kHidden;
        total = b3 + 1;
    }
};

// Forward pass for rows [0, n): y[r]; also stores the hidden activations
// when h1/h2 are non-null (needed by the backward pass).
__global__ void __launch_bounds__(256)
    mlp_forward_kernel(const float *__restrict__ params, int in, const float *__restrict__ X,
                       int n, float *__restrict__ y, float *__restrict__ h1,
                       float *__restrict__ h2) {
    extern __shared__ float sm[];
    const int nw1 = in * kHidden;
    float *W1 = sm, *B1 = W1 + nw1, *W2 = B1 + kHidden, *B2 = W2 + kHidden * kHidden,
          *W3 = B2 + kHidden;
    float *act = W3 + kHidden + 1;  // per warp: 2 x kHidden
    const int total = nw1 + kHidden + kHidden * kHidden + kHidden + kHidden + 1;
    for (int i = threadIdx.x; i < total; i += blockDim.x) sm[i] = params[i];
    __syncthreads();
    const float b3 = W3[kHidden];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *a1 = act + warp * 2 * kHidden, *a2 = a1 + kHidden;
    for (int r = blockIdx.x * kRowsPerCta + warp; r < n; r += gridDim.x * kRowsPerCta) {
        const float *x = X + (int64_t)r * in;
        for (int u = lane; u < kHidden; u += 32) {
            float s = B1[u];
            for (int f = 0; f < in; f++) s += x[f] * W1[f * kHidden + u];
            a1[u] = s > 0.f ? s : 0.f;
        }
        __syncwarp();
        for (int u = lane; u < kHidden; u += 32) {
            float s = B2[u];
            for (int k = 0; k < kHidden; k++) s += a1[k] * W2[k * kHidden + u];
            a2[u] = s > 0.f ? s : 0.f;
        }
        __syncwarp();
        float part = a2[lane] * W3[lane] + a2[lane + 32] * W3[lane + 32];
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) y[r] = part + b3;
        if (h1)
            for (int u = lane; u < kHidden; u += 32) {
                h1[(int64_t)r * kHidden + u] = a1[u];
                h2[(int64_t)r * kHidden + u] = a2[u];
            }
        __syncwarp();
    }
}

// Backward, step 1 (one warp per row): the loss gradients at the output and
// at both hidden layers' pre-activations, for L = mean_r (y_r - t_r)^2:
//   dy_r = 2 (y_r - t_r) / n,  d2 = dy w3 . [h2 > 0],  d1 = (d2 W2^T) . [h1 > 0]
__global__ void __launch_bounds__(256)
    mlp_delta_kernel(const float *__restrict__ params, int in, const float *__restrict__ T,
                     const float *__restrict__ y, const float *__restrict__ h1,
                     const float *__restrict__ h2, int n, float *__restrict__ dyo,
                     float *__restrict__ d2o, float *__restrict__ d1o) {
    extern __shared__ float sm[];
    const int nw1 = in * kHidden;
    float *W2 = sm, *W3 = W2 + kHidden * kHidden;
    for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x)
        W2[i] = params[nw1 + kHidden + i];
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x)
        W3[i] = params[nw1 + kHidden + kHidden * kHidden + kHidden + i];
    __syncthreads();
    float *scr = W3 + kHidden;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *d2 = scr + warp * kHidden;
    const float scale = 2.f / (float)n;
    for (int r = blockIdx.x * kRowsPerCta + warp; r < n; r += gridDim.x * kRowsPerCta) {
        const float dy = scale * (y[r] - T[r]);
        const float *a1 = h1 + (int64_t)r * kHidden, *a2 = h2 + (int64_t)r * kHidden;
        for (int u = lane; u < kHidden; u += 32) {
            const float v = a2[u] > 0.f ? dy * W3[u] : 0.f;
            d2[u] = v;
            d2o[(int64_t)r * kHidden + u] = v;
        }
        __syncwarp();
        for (int k = lane; k < kHidden; k += 32) {
            float s = 0.f;
            for (int u = 0; u < kHidden; u++) s += d2[u] * W2[k * kHidden + u];
            d1o[(int64_t)r * kHidden + k] = a1[k] > 0.f ? s : 0.f;
        }
        if (lane == 0) dyo[r] = dy;
        __syncwarp();
    }
}

// Backward, step 2 (one thread per parameter, rows summed in order, so the
// result is deterministic): dW1 = X^T d1, db1 = sum d1, dW2 = h1^T d2,
// db2 = sum d2, dw3 = h2^T dy, db3 = sum dy.  Written (not added) to grad.
__global__ void mlp_param_grad_kernel(int in, const float *__restrict__ X,
                                      const float *__restrict__ h1,
                                      const float *__restrict__ h2,
                                      const float *__restrict__ dy,
                                      const float *__restrict__ d2,
                                      const float *__restrict__ d1, int n,
                                      float *__restrict__ grad) {
    const int nw1 = in * kHidden;
    const int total = nw1 + kHidden + kHidden * kHidden + kHidden + kHidden + 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    float s = 0.f;
    if (i < nw1) {
        const int f = i / kHidden, u = i % kHidden;
        for (int r = 0; r < n; r++) s += X[(int64_t)r * in + f] * d1[(int64_t)r * kHidden + u];
    } else if (i < nw1 + kHidden) {
        const int u = i - nw1;
        for (int r = 0; r < n; r++) s += d1[(int64_t)r * kHidden + u];
    } else if (i < nw1 + kHidden + kHidden * kHidden) {
        const int j = i - nw1 - kHidden, k = j / kHidden, u = j % kHidden;
        for (int r = 0; r < n; r++) s += h1[(int64_t)r * kHidden + k] * d2[(int64_t)r * kHidden + u];
    } else if (i < nw1 + 2 * kHidden + kHidden * kHidden) {
        const int u = i - nw1 - kHidden - kHidden * kHidden;
        for (int r = 0; r < n; r++) s += d2[(int64_t)r * kHidden + u];
    } else if (i < total - 1) {
        const int u = i - nw1 - 2 * kHidden - kHidden * kHidden;
        for (int r = 0; r < n; r++) s += h2[(int64_t)r * kHidden + u] * dy[r];
    } else {
        for (int r = 0; r < n; r++) s += dy[r];
    }
    grad[i] = s;
}

// Adam (Kingma & Ba 2015) with bias correction; step is 1-based.
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int n, float lr,
                            float b1, float b2, float eps, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.f - powf(b1, (float)step));
    const float vh = vi / (1.f - powf(b2, (float)step));
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void sq_err_kernel(const float *y, const float *t, int n, float *out) {
    float s = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float d = y[i] - t[i];
        s += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

int grid_for(int n) {
    int g = (n + kRowsPerCta - 1) / kRowsPerCta;
    return g < 1 ? 1 : (g > 1184 ? 1184 : g);
}

size_t fwd_smem(int in) { return sizeof(float) * (in * kHidden + 3 * kHidden + kHidden * kHidden + 1 + 8 * 2 * kHidden); }
size_t delta_smem() { return sizeof(float) * (kHidden * kHidden + kHidden + 8 * kHidden); }

// One backward pass over rows [0, n) given the forward activations: writes
// the full-batch gradient into grad.
void backward(const float *params, int in, const float *X, const float *T, const float *y,
              const float *h1, const float *h2, int n, float *dy, float *d2, float *d1,
              float *grad, int total) {
    mlp_delta_kernel<<<grid_for(n), 256, delta_smem()>>>(params, in, T, y, h1, h2, n, dy, d2,
                                                          d1);
    mlp_param_grad_kernel<<<(total + 127) / 128, 128>>>(in, X, h1, h2, dy, d2, d1, n, grad);
}

}  // namespace

struct gat_mlp {
    Shape shape{1};
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    int step = 0;
    ~gat_mlp() {
        cudaFree(params);
        cudaFree(grad);
        cudaFree(m);
        cudaFree(v);
    }
};

namespace {
int mlp_fail(int code, const std::string &msg) {
    g_mlp_err = msg;
    return code;
}
int cerr(cudaError_t e, const char *what) {
    return mlp_fail(GAT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, n > 0 ? n : 4); }
    float *f() { return static_cast<float *>(p); }
};

cudaError_t set_attrs(int in) {
    cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fwd_smem(in));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(mlp_delta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)delta_smem());
}

}  // namespace

extern "C" {

const char *gat_mlp_last_error(void) { return g_mlp_err.c_str(); }

int gat_mlp_create(int in_features, uint64_t seed, gat_mlp **out) {
    if (!out || in_features < 1 || in_features > kMaxIn)
        return mlp_fail(GAT_ERR_ARGUMENT, "in_features must be in [1, 64]");
    auto *net = new gat_mlp;
    net->shape = Shape(in_features);
    const int P = net->shape.total;
    cudaError_t e;
    if ((e = cudaMalloc(&net->params, sizeof(float) * P)) != cudaSuccess ||
        (e = cudaMalloc(&net->grad, sizeof(float) * P)) != cudaSuccess ||
        (e = cudaMalloc(&net->m, sizeof(float) * P)) != cudaSuccess ||
        (e = cudaMalloc(&net->v, sizeof(float) * P)) != cudaSuccess) {
        delete net;
        return cerr(e, "mlp allocation");
    }
    // He-uniform initial weights, zero biases (host generated, seeded).
    std::vector<float> h(P, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int count) {
        const float lim = std::sqrt(6.f / (float)fan_in);
        std::uniform_real_distribution<float> d(-lim, lim);
        for (int i = 0; i < count; i++) h[off + i] = d(rng);
    };
    const Shape &s = net->shape;
    fill(s.w1, s.in, s.in * kHidden);
    fill(s.w2, kHidden, kHidden * kHidden);
    fill(s.w3, kHidden, kHidden);
    if ((e = cudaMemcpy(net->params, h.data(), sizeof(float) * P, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemset(net->m, 0, sizeof(float) * P)) != cudaSuccess ||
        (e = cudaMemset(net->v, 0, sizeof(float) * P)) != cudaSuccess ||
        (e = set_attrs(s.in)) != cudaSuccess) {
        delete net;
        return cerr(e, "mlp init");
    }
    *out = net;
    return GAT_OK;
}

void gat_mlp_free(gat_mlp *net) { delete net; }

int gat_mlp_num_params(const gat_mlp *net) { return net ? net->shape.total : 0; }

int gat_mlp_get_params(const gat_mlp *net, float *out, int n) {
    if (!net || !out || n < net->shape.total) return mlp_fail(GAT_ERR_ARGUMENT, "bad buffer");
    cudaError_t e = cudaMemcpy(out, net->params, sizeof(float) * net->shape.total,
                               cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? GAT_OK : cerr(e, "get params");
}

int gat_mlp_set_params(gat_mlp *net, const float *in, int n) {
    if (!net || !in || n < net->shape.total) return mlp_fail(GAT_ERR_ARGUMENT, "bad buffer");
    cudaError_t e = cudaMemcpy(net->params, in, sizeof(float) * net->shape.total,
                               cudaMemcpyHostToDevice);
    net->step = 0;
    if (e == cudaSuccess) e = cudaMemset(net->m, 0, sizeof(float) * net->shape.total);
    if (e == cudaSuccess) e = cudaMemset(net->v, 0, sizeof(float) * net->shape.total);
    return e == cudaSuccess ? GAT_OK : cerr(e, "set params");
}

int gat_mlp_predict(const gat_mlp *net, const float *X, int n, float *y) {
    if (!net || !X || !y || n < 0) return mlp_fail(GAT_ERR_ARGUMENT, "bad arguments");
    if (n == 0) return GAT_OK;
    const int in = net->shape.in;
    DevBuf dx, dy;
    cudaError_t e;
    if ((e = dx.alloc(sizeof(float) * n * in)) != cudaSuccess ||
        (e = dy.alloc(sizeof(float) * n)) != cudaSuccess)
        return cerr(e, "predict buffers");
    cudaMemcpy(dx.p, X, sizeof(float) * n * in, cudaMemcpyHostToDevice);
    mlp_forward_kernel<<<grid_for(n), 256, fwd_smem(in)>>>(net->params, in, dx.f(), n, dy.f(),
                                                           nullptr, nullptr);
    if ((e = cudaGetLastError()) != cudaSuccess) return cerr(e, "forward");
    e = cudaMemcpy(y, dy.p, sizeof(float) * n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? GAT_OK : cerr(e, "predict");
}

// Mean squared error and its gradient over all n rows (no update), for
// checking the kernels against a CPU reference.
int gat_mlp_gradient(const gat_mlp *net, const float *X, const float *T, int n,
                     float *grad_out, float *loss) {
    if (!net || !X || !T || !grad_out || n <= 0) return mlp_fail(GAT_ERR_ARGUMENT, "bad arguments");
    const int in = net->shape.in, P = net->shape.total;
    DevBuf dx, dt, dy, h1, h2, g, l, ddy, dd2, dd1;
    cudaError_t e;
    if ((e = dx.alloc(sizeof(float) * n * in)) != cudaSuccess ||
        (e = dt.alloc(sizeof(float) * n)) != cudaSuccess ||
        (e = dy.alloc(sizeof(float) * n)) != cudaSuccess ||
        (e = h1.alloc(sizeof(float) * n * kHidden)) != cudaSuccess ||
        (e = h2.alloc(sizeof(float) * n * kHidden)) != cudaSuccess ||
        (e = g.alloc(sizeof(float) * P)) != cudaSuccess ||
        (e = l.alloc(sizeof(float))) != cudaSuccess ||
        (e = ddy.alloc(sizeof(float) * n)) != cudaSuccess ||
        (e = dd2.alloc(sizeof(float) * n * kHidden)) != cudaSuccess ||
        (e = dd1.alloc(sizeof(float) * n * kHidden)) != cudaSuccess)
        return cerr(e, "gradient buffers");
    cudaMemcpy(dx.p, X, sizeof(float) * n * in, cudaMemcpyHostToDevice);
    cudaMemcpy(dt.p, T, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemset(g.p, 0, sizeof(float) * P);
    cudaMemset(l.p, 0, sizeof(float));
    mlp_forward_kernel<<<grid_for(n), 256, fwd_smem(in)>>>(net->params, in, dx.f(), n, dy.f(),
                                                           h1.f(), h2.f());
    backward(net->params, in, dx.f(), dt.f(), dy.f(), h1.f(), h2.f(), n, ddy.f(), dd2.f(),
             dd1.f(), g.f(), P);
    sq_err_kernel<<<32, 256>>>(dy.f(), dt.f(), n, l.f());
    if ((e = cudaGetLastError()) != cudaSuccess) return cerr(e, "gradient kernels");
    float s = 0.f;
    if ((e = cudaMemcpy(grad_out, g.p, sizeof(float) * P, cudaMemcpyDeviceToHost)) !=
            cudaSuccess ||
        (e = cudaMemcpy(&s, l.p, sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cerr(e, "gradient copy");
    if (loss) *loss = s / (float)n;
    return GAT_OK;
}

// Mini-batch Adam training on (X, T); rows are visited in a seeded random
// order each epoch.  *final_loss (may be null) is the full-data MSE after
// training.
int gat_mlp_train(gat_mlp *net, const float *X, const float *T, int n, int epochs,
                  int batch, float lr, uint64_t seed, float *final_loss) {
    if (!net || !X || !T || n <= 0 || epochs < 0 || batch <= 0)
        return mlp_fail(GAT_ERR_ARGUMENT, "bad arguments");
    const int in = net->shape.in, P = net->shape.total;
    DevBuf dx, dt, dxb, dtb, dy, h1, h2, l, ddy, dd2, dd1;
    cudaError_t e;
    if ((e = ddy.alloc(sizeof(float) * n)) != cudaSuccess ||
        (e = dd2.alloc(sizeof(float) * n * kHidden)) != cudaSuccess ||
        (e = dd1.alloc(sizeof(float) * n * kHidden)) != cudaSuccess ||
        (e = dx.alloc(sizeof(float) * n * in)) != cudaSuccess ||
        (e = dt.alloc(sizeof(float) * n)) != cudaSuccess ||
        (e = dxb.alloc(sizeof(float) * n * in)) != cudaSuccess ||
        (e = dtb.alloc(sizeof(float) * n)) != cudaSuccess ||
        (e = dy.alloc(sizeof(float) * n)) != cudaSuccess ||
        (e = h1.alloc(sizeof(float) * n * kHidden)) != cudaSuccess ||
        (e = h2.alloc(sizeof(float) * n * kHidden)) != cudaSuccess ||
        (e = l.alloc(sizeof(float))) != cudaSuccess)
        return cerr(e, "train buffers");
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::mt19937_64 rng(seed);
    std::vector<float> xs(size_t(n) * in), ts(n);
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(order.begin(), order.end(), rng);
        for (int i = 0; i < n; i++) {
            std::memcpy(&xs[size_t(i) * in], &X[size_t(order[i]) * in], sizeof(float) * in);
            ts[i] = T[order[i]];
        }
        cudaMemcpy(dxb.p, xs.data(), sizeof(float) * n * in, cudaMemcpyHostToDevice);
        cudaMemcpy(dtb.p, ts.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
        for (int b0 = 0; b0 < n; b0 += batch) {
            const int nb = std::min(batch, n - b0);
            const float *xb = dxb.f() + size_t(b0) * in;
            const float *tb = dtb.f() + b0;
            mlp_forward_kernel<<<grid_for(nb), 256, fwd_smem(in)>>>(net->params, in, xb, nb,
                                                                    dy.f(), h1.f(), h2.f());
            backward(net->params, in, xb, tb, dy.f(), h1.f(), h2.f(), nb, ddy.f(), dd2.f(),
                     dd1.f(), net->grad, P);
            net->step++;
            adam_kernel<<<(P + 255) / 256, 256>>>(net->params, net->grad, net->m, net->v, P, lr,
                                                  0.9f, 0.999f, 1e-8f, net->step);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cerr(e, "training kernels");
    }
    if (final_loss) {
        cudaMemcpy(dx.p, X, sizeof(float) * n * in, cudaMemcpyHostToDevice);
        cudaMemcpy(dt.p, T, sizeof(float) * n, cudaMemcpyHostToDevice);
        cudaMemset(l.p, 0, sizeof(float));
        mlp_forward_kernel<<<grid_for(n), 256, fwd_smem(in)>>>(net->params, in, dx.f(), n,
                                                               dy.f(), nullptr, nullptr);
        sq_err_kernel<<<32, 256>>>(dy.f(), dt.f(), n, l.f());
        float s = 0.f;
        if ((e = cudaMemcpy(&s, l.p, sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cerr(e, "final loss");
        *final_loss = s / (float)n;
    }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cerr(e, "train");
    return GAT_OK;
}

}  // extern "C"
