// The firing predictor's MLP (9 -> 64 -> 64 -> 1, ReLU): deterministic
// initialisation, batched forward pass, mean-squared-error backward pass and
// Adam training, all as hand-written CUDA kernels. Inference inside the
// simulation step lives in step.cu (one warp per population).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>
#include <vector>

#include "engine.h"
#include "netgen.h"

namespace bsim {
int record_error(int code, const std::string &msg);
}
using namespace bsim;

namespace {

constexpr int IN = BSIM_MLP_IN, H = BSIM_MLP_HIDDEN, NP = BSIM_MLP_PARAMS;
constexpr int OFF_W1 = 0, OFF_B1 = H * IN, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H, OFF_W3 = OFF_B2 + H,
              OFF_B3 = OFF_W3 + H;
static_assert(OFF_B3 + 1 == NP, "parameter layout");

int fail(int code, const std::string &m, cudaError_t st = cudaSuccess)
{
    return record_error(code, st == cudaSuccess ? m : m + ": " + cudaGetErrorString(st));
}

// Forward pass: thread per sample, parameters staged in shared memory.
__global__ void mlp_forward_kernel(const float *params, const float *x, int64_t n, float *y_out)
{
    __shared__ float P[NP];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xi[IN], h1[H];
    for (int k = 0; k < IN; k++) xi[k] = x[i * IN + k];
    for (int u = 0; u < H; u++) {
        float s = P[OFF_B1 + u];
        for (int k = 0; k < IN; k++) s = fmaf(P[OFF_W1 + u * IN + k], xi[k], s);
        h1[u] = fmaxf(s, 0.0f);
    }
    float y = P[OFF_B3];
    for (int u = 0; u < H; u++) {
        float s = P[OFF_B2 + u];
        for (int k = 0; k < H; k++) s = fmaf(P[OFF_W2 + u * H + k], h1[k], s);
        y = fmaf(P[OFF_W3 + u], fmaxf(s, 0.0f), y);
    }
    y_out[i] = y;
}

// Backward pass over tiles of GT samples, one thread per sample for the
// forward and the per-sample error terms (kept in shared memory, rows padded to
// 65 words against bank conflicts), then one thread per group of parameters
// summing its gradient over the tile's samples: one global atomic per parameter
// and tile instead of one shared atomic per parameter and sample.
constexpr int GT = 64, RS = H + 1;
constexpr size_t GRAD_SMEM = sizeof(float) * (NP + 4 * GT * RS + GT * IN + GT);

__global__ void __launch_bounds__(GT) mlp_grad_kernel(const float *params, const float *x, const float *y_target,
                                                       int64_t n, float *grad, double *loss_acc)
{
    extern __shared__ float sm[];
    float *P = sm;
    float *s_h1 = P + NP, *s_h2 = s_h1 + GT * RS, *s_dz2 = s_h2 + GT * RS, *s_dz1 = s_dz2 + GT * RS;
    float *s_x = s_dz1 + GT * RS, *s_dy = s_x + GT * IN;
    for (int i = threadIdx.x; i < NP; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int t = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * GT + t;
    float *h1 = s_h1 + t * RS, *h2 = s_h2 + t * RS, *dz2 = s_dz2 + t * RS, *dz1 = s_dz1 + t * RS;
    float *xi = s_x + t * IN;
    double sq = 0.0;
    if (i < n) {
        for (int k = 0; k < IN; k++) xi[k] = x[i * IN + k];
        for (int u = 0; u < H; u++) {
            float s = P[OFF_B1 + u];
            for (int k = 0; k < IN; k++) s = fmaf(P[OFF_W1 + u * IN + k], xi[k], s);
            h1[u] = fmaxf(s, 0.0f);
        }
        float y = P[OFF_B3];
        for (int u = 0; u < H; u++) {
            float s = P[OFF_B2 + u];
            for (int k = 0; k < H; k++) s = fmaf(P[OFF_W2 + u * H + k], h1[k], s);
            h2[u] = fmaxf(s, 0.0f);
            y = fmaf(P[OFF_W3 + u], h2[u], y);
        }
        const float e = y - y_target[i];
        sq = (double)e * (double)e;
        const float dy = 2.0f * e / (float)n;
        s_dy[t] = dy;
        for (int u = 0; u < H; u++) dz2[u] = h2[u] > 0.0f ? dy * P[OFF_W3 + u] : 0.0f;
        for (int k = 0; k < H; k++) {
            float d = 0.0f;
            for (int u = 0; u < H; u++) d = fmaf(dz2[u], P[OFF_W2 + u * H + k], d);
            dz1[k] = h1[k] > 0.0f ? d : 0.0f;
        }
    } else {  // samples past the end contribute nothing
        s_dy[t] = 0.0f;
        for (int k = 0; k < IN; k++) xi[k] = 0.0f;
        for (int u = 0; u < H; u++) h1[u] = h2[u] = dz2[u] = dz1[u] = 0.0f;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if ((t & 31) == 0 && sq != 0.0) atomicAdd(loss_acc, sq / (double)n);
    __syncthreads();
    // gradients of this tile, parameter by parameter
    for (int j = t; j < NP; j += GT) {
        float g = 0.0f;
        if (j < OFF_B1) {  // W1[u][k]
            const int u = j / IN, k = j % IN;
            for (int b = 0; b < GT; b++) g = fmaf(s_dz1[b * RS + u], s_x[b * IN + k], g);
        } else if (j < OFF_W2) {  // b1[u]
            for (int b = 0; b < GT; b++) g += s_dz1[b * RS + (j - OFF_B1)];
        } else if (j < OFF_B2) {  // W2[u][k]
            const int u = (j - OFF_W2) / H, k = (j - OFF_W2) % H;
            for (int b = 0; b < GT; b++) g = fmaf(s_dz2[b * RS + u], s_h1[b * RS + k], g);
        } else if (j < OFF_W3) {  // b2[u]
            for (int b = 0; b < GT; b++) g += s_dz2[b * RS + (j - OFF_B2)];
        } else if (j < OFF_B3) {  // W3[u]
            for (int b = 0; b < GT; b++) g = fmaf(s_dy[b], s_h2[b * RS + (j - OFF_W3)], g);
        } else {  // b3
            for (int b = 0; b < GT; b++) g += s_dy[b];
        }
        if (g != 0.0f) atomicAdd(&grad[j], g);
    }
}

// Launches the backward pass (the shared-memory size needs the opt-in once).
cudaError_t launch_grad(const float *p, const float *x, const float *y, int64_t n, float *g, double *l)
{
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t st = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)GRAD_SMEM);
        if (st != cudaSuccess) return st;
        attr_set = true;
    }
    mlp_grad_kernel<<<(unsigned)((n + GT - 1) / GT), GT, GRAD_SMEM>>>(p, x, y, n, g, l);
    return cudaGetLastError();
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, float lr, float b1t, float b2t)
{
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        m[i] = b1 * m[i] + (1.0f - b1) * gi;
        v[i] = b2 * v[i] + (1.0f - b2) * gi * gi;
        const float mh = m[i] / (1.0f - b1t), vh = v[i] / (1.0f - b2t);
        p[i] -= lr * mh / (sqrtf(vh) + eps);
    }
}

__global__ void gather_rows(const float *x, const float *y, const int64_t *idx, int64_t n, float *xb, float *yb)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = idx[i];
        for (int k = 0; k < IN; k++) xb[i * IN + k] = x[r * IN + k];
        yb[i] = y[r];
    }
}

struct DevBuf {
    std::vector<void *> p;
    ~DevBuf()
    {
        for (void *q : p) cudaFree(q);
    }
    template <typename T>
    cudaError_t get(T **out, size_t count)
    {
        cudaError_t st = cudaMalloc((void **)out, sizeof(T) * (count ? count : 1));
        if (st == cudaSuccess) p.push_back(*out);
        return st;
    }
};

}  // namespace

extern "C" int bsim_mlp_init(float *params, uint64_t seed)
{
    if (!params) return fail(BSIM_ERR_ARG, "bsim_mlp_init: null params");
    memset(params, 0, sizeof(float) * NP);
    auto fill = [&](int off, int fan_in, int fan_out, int count, uint64_t salt) {
        const float a = sqrtf(6.0f / (float)(fan_in + fan_out));
        for (int i = 0; i < count; i++) {
            const float u = unit24((uint32_t)(hash3(seed, salt, (uint64_t)i) >> 40));
            params[off + i] = (2.0f * u - 1.0f) * a;
        }
    };
    fill(OFF_W1, IN, H, H * IN, 1);
    fill(OFF_W2, H, H, H * H, 2);
    fill(OFF_W3, H, 1, H, 3);
    return BSIM_OK;
}

extern "C" int bsim_mlp_forward(const float *params, const float *x, int64_t n, float *y)
{
    if (!params || n < 0 || (n > 0 && (!x || !y))) return fail(BSIM_ERR_ARG, "bsim_mlp_forward: invalid arguments");
    if (n == 0) return BSIM_OK;
    DevBuf b;
    float *dp, *dx, *dy;
    cudaError_t st;
    if ((st = b.get(&dp, NP)) || (st = b.get(&dx, n * IN)) || (st = b.get(&dy, n)))
        return fail(BSIM_ERR_NOMEM, "bsim_mlp_forward: allocation", st);
    cudaMemcpy(dp, params, sizeof(float) * NP, cudaMemcpyHostToDevice);
    cudaMemcpy(dx, x, sizeof(float) * n * IN, cudaMemcpyHostToDevice);
    mlp_forward_kernel<<<(unsigned)((n + 127) / 128), 128>>>(dp, dx, n, dy);
    st = cudaMemcpy(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (st != cudaSuccess) return fail(BSIM_ERR_CUDA, "bsim_mlp_forward", st);
    return BSIM_OK;
}

extern "C" int bsim_mlp_grad(const float *params, const float *x, const float *y_target, int64_t n, float *grad,
                             float *loss)
{
    if (!params || n <= 0 || !x || !y_target || !grad) return fail(BSIM_ERR_ARG, "bsim_mlp_grad: invalid arguments");
    DevBuf b;
    float *dp, *dx, *dt, *dg;
    double *dl;
    cudaError_t st;
    if ((st = b.get(&dp, NP)) || (st = b.get(&dx, n * IN)) || (st = b.get(&dt, n)) || (st = b.get(&dg, NP)) ||
        (st = b.get(&dl, 1)))
        return fail(BSIM_ERR_NOMEM, "bsim_mlp_grad: allocation", st);
    cudaMemcpy(dp, params, sizeof(float) * NP, cudaMemcpyHostToDevice);
    cudaMemcpy(dx, x, sizeof(float) * n * IN, cudaMemcpyHostToDevice);
    cudaMemcpy(dt, y_target, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemset(dg, 0, sizeof(float) * NP);
    cudaMemset(dl, 0, sizeof(double));
    if ((st = launch_grad(dp, dx, dt, n, dg, dl)) != cudaSuccess) return fail(BSIM_ERR_CUDA, "bsim_mlp_grad", st);
    double l = 0;
    st = cudaMemcpy(grad, dg, sizeof(float) * NP, cudaMemcpyDeviceToHost);
    if (st == cudaSuccess) st = cudaMemcpy(&l, dl, sizeof(double), cudaMemcpyDeviceToHost);
    if (st != cudaSuccess) return fail(BSIM_ERR_CUDA, "bsim_mlp_grad", st);
    if (loss) *loss = (float)l;
    return BSIM_OK;
}

extern "C" int bsim_mlp_train(float *params, const float *x, const float *y_target, int64_t n, int32_t epochs,
                              int32_t batch, float lr, uint64_t seed, float *final_loss)
{
    if (!params || n <= 0 || !x || !y_target || epochs < 0 || batch <= 0 || !(lr > 0))
        return fail(BSIM_ERR_ARG, "bsim_mlp_train: invalid arguments");
    DevBuf b;
    float *dp, *dx, *dt, *dg, *dm, *dv, *xb, *yb;
    int64_t *didx;
    double *dl;
    cudaError_t st;
    const int64_t bs = std::min<int64_t>(batch, n);
    if ((st = b.get(&dp, NP)) || (st = b.get(&dx, n * IN)) || (st = b.get(&dt, n)) || (st = b.get(&dg, NP)) ||
        (st = b.get(&dm, NP)) || (st = b.get(&dv, NP)) || (st = b.get(&xb, bs * IN)) || (st = b.get(&yb, bs)) ||
        (st = b.get(&didx, n)) || (st = b.get(&dl, 1)))
        return fail(BSIM_ERR_NOMEM, "bsim_mlp_train: allocation", st);
    cudaMemcpy(dp, params, sizeof(float) * NP, cudaMemcpyHostToDevice);
    cudaMemcpy(dx, x, sizeof(float) * n * IN, cudaMemcpyHostToDevice);
    cudaMemcpy(dt, y_target, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemset(dm, 0, sizeof(float) * NP);
    cudaMemset(dv, 0, sizeof(float) * NP);
    std::vector<int64_t> idx(n);
    for (int64_t i = 0; i < n; i++) idx[i] = i;
    float b1t = 1.0f, b2t = 1.0f;
    int64_t step = 0;
    for (int ep = 0; ep < epochs; ep++) {
        // deterministic shuffle (Fisher-Yates on the seeded hash)
        for (int64_t i = n - 1; i > 0; i--) {
            const int64_t j = (int64_t)(hash3(seed, (uint64_t)ep, (uint64_t)i) % (uint64_t)(i + 1));
            std::swap(idx[i], idx[j]);
        }
        cudaMemcpy(didx, idx.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice);
        for (int64_t b0 = 0; b0 + bs <= n; b0 += bs) {
            gather_rows<<<64, 256>>>(dx, dt, didx + b0, bs, xb, yb);
            cudaMemsetAsync(dg, 0, sizeof(float) * NP);
            cudaMemsetAsync(dl, 0, sizeof(double));
            if ((st = launch_grad(dp, xb, yb, bs, dg, dl)) != cudaSuccess) return fail(BSIM_ERR_CUDA, "bsim_mlp_train", st);
            step++;
            b1t *= 0.9f;
            b2t *= 0.999f;
            adam_kernel<<<(NP + 255) / 256, 256>>>(dp, dg, dm, dv, lr, b1t, b2t);
        }
    }
    // loss over the whole set
    cudaMemset(dg, 0, sizeof(float) * NP);
    cudaMemset(dl, 0, sizeof(double));
    if ((st = launch_grad(dp, dx, dt, n, dg, dl)) != cudaSuccess) return fail(BSIM_ERR_CUDA, "bsim_mlp_train", st);
    double l = 0;
    st = cudaMemcpy(params, dp, sizeof(float) * NP, cudaMemcpyDeviceToHost);
    if (st == cudaSuccess) st = cudaMemcpy(&l, dl, sizeof(double), cudaMemcpyDeviceToHost);
    if (st != cudaSuccess) return fail(BSIM_ERR_CUDA, "bsim_mlp_train", st);
    if (final_loss) *final_loss = (float)l;
    return BSIM_OK;
}
