// mlp.cu -- the learned matching-order cost model: a small FP32 MLP
// (in -> H -> H -> 1, ReLU) trained and evaluated by hand-written kernels.
//
// It predicts log(1 + |L_i|), the size of trie level i, from per-step
// features of a candidate order; the order search (order_search.cpp) sums
// the predictions into a work estimate and keeps the cheapest order.
//
// Training is full-batch or mini-batch Adam on the mean squared error.  One
// fused kernel runs forward + backward for a slice of samples per block,
// keeping both hidden activations in shared memory, and accumulates the
// block's gradient in shared memory before one atomic add per parameter.
// Sizes are tiny (in <= 32, H = 64), so the kernels are latency-bound FP32
// CUDA-core work; tensor cores are not worth their setup here.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mlp.hpp"

namespace cuts {

#define MCK(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return set_error(CUTS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr int kH = MLP_HIDDEN;
constexpr int kMaxIn = MLP_MAX_IN;
constexpr int kThreads = 256;          // 4 samples in flight per block, 64 threads each
constexpr int kPerBlock = kThreads / kH;

// parameter layout: W1[H][in] b1[H] W2[H][H] b2[H] W3[H] b3
__host__ __device__ inline int n_params(int in) { return kH * in + kH + kH * kH + kH + kH + 1; }

struct Layout {
    int w1, b1, w2, b2, w3, b3, total;
};
__host__ __device__ inline Layout layout(int in) {
    Layout L;
    L.w1 = 0;
    L.b1 = L.w1 + kH * in;
    L.w2 = L.b1 + kH;
    L.b2 = L.w2 + kH * kH;
    L.w3 = L.b2 + kH;
    L.b3 = L.w3 + kH;
    L.total = L.b3 + 1;
    return L;
}

// Forward (and, when grad != nullptr, backward) over samples [0, n).
// loss_acc += sum (y - t)^2; grad += d(mean loss)/d(params).
__global__ void __launch_bounds__(kThreads)
k_mlp(const float *__restrict__ params, int in, const float *__restrict__ X,
      const float *__restrict__ T, int n, float *__restrict__ Y, float *__restrict__ grad,
      float *__restrict__ loss_acc) {
    extern __shared__ float sm[];
    const Layout L = layout(in);
    float *P = sm;                        // params
    float *G = P + L.total;               // block gradient (only when training)
    float *x = G + (grad ? L.total : 0);  // [kPerBlock][kMaxIn]
    float *h1 = x + kPerBlock * kMaxIn;   // [kPerBlock][H]
    float *h2 = h1 + kPerBlock * kH;      // [kPerBlock][H]
    float *dh2 = h2 + kPerBlock * kH;     // [kPerBlock][H]
    float *red = dh2 + kPerBlock * kH;    // [kPerBlock][2]
    for (int i = threadIdx.x; i < L.total; i += blockDim.x) {
        P[i] = params[i];
        if (grad) G[i] = 0.f;
    }
    __syncthreads();
    const int s = threadIdx.x / kH;   // sample slot in the block
    const int j = threadIdx.x % kH;   // hidden unit
    const int lane = threadIdx.x & 31;
    float lsum = 0.f;
    const float inv_n = 1.f / float(max(n, 1));
    for (int base = blockIdx.x * kPerBlock; base < n; base += gridDim.x * kPerBlock) {
        const int r = base + s;
        const bool valid = r < n;
        if (j < in) x[s * kMaxIn + j] = valid ? X[size_t(r) * in + j] : 0.f;
        __syncthreads();
        // layer 1
        float a = P[L.b1 + j];
        for (int f = 0; f < in; ++f) a += P[L.w1 + j * in + f] * x[s * kMaxIn + f];
        const float z1 = fmaxf(a, 0.f);
        h1[s * kH + j] = z1;
        __syncthreads();
        // layer 2
        float b = P[L.b2 + j];
        for (int i = 0; i < kH; ++i) b += P[L.w2 + j * kH + i] * h1[s * kH + i];
        const float z2 = fmaxf(b, 0.f);
        h2[s * kH + j] = z2;
        // output: two warps per sample slot reduce w3 . h2
        float o = P[L.w3 + j] * z2;
        #pragma unroll
        for (int d = 16; d; d >>= 1) o += __shfl_xor_sync(0xffffffffu, o, d);
        if (lane == 0) red[s * 2 + (j >> 5)] = o;
        __syncthreads();
        const float y = red[s * 2] + red[s * 2 + 1] + P[L.b3];
        if (valid && j == 0 && Y) Y[r] = y;
        float dy = 0.f;
        if (valid && T) {
            const float e = y - T[r];
            if (j == 0) lsum += e * e;
            dy = 2.f * e * inv_n;
        }
        if (grad && valid) {
            // output layer
            atomicAdd(&G[L.w3 + j], dy * z2);
            if (j == 0) atomicAdd(&G[L.b3], dy);
            const float d2 = z2 > 0.f ? dy * P[L.w3 + j] : 0.f;
            dh2[s * kH + j] = d2;
            atomicAdd(&G[L.b2 + j], d2);
            for (int i = 0; i < kH; ++i) atomicAdd(&G[L.w2 + j * kH + i], d2 * h1[s * kH + i]);
        }
        __syncthreads();
        if (grad && valid) {
            // hidden unit j of layer 1
            float d1 = 0.f;
            for (int i = 0; i < kH; ++i) d1 += P[L.w2 + i * kH + j] * dh2[s * kH + i];
            d1 = z1 > 0.f ? d1 : 0.f;
            atomicAdd(&G[L.b1 + j], d1);
            for (int f = 0; f < in; ++f) atomicAdd(&G[L.w1 + j * in + f], d1 * x[s * kMaxIn + f]);
        }
        __syncthreads();
    }
    if (grad) {
        for (int i = threadIdx.x; i < L.total; i += blockDim.x)
            if (G[i] != 0.f) atomicAdd(&grad[i], G[i]);
    }
    if (loss_acc && j == 0 && lsum != 0.f) atomicAdd(loss_acc, lsum);
}

// Adam (Kingma & Ba 2015) with bias correction.
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

size_t smem_bytes(int in, bool train) {
    const int total = layout(in).total;
    return sizeof(float) * (size_t(total) * (train ? 2 : 1) + kPerBlock * kMaxIn + 3 * kPerBlock * kH +
                            2 * kPerBlock);
}

}  // namespace

int mlp_param_count(int in) { return n_params(in); }

int Mlp::create(int in_dim, uint64_t seed, int dev) {
    if (in_dim < 1 || in_dim > kMaxIn) return set_error(CUTS_ERR_ARG, "mlp input dim out of range");
    in = in_dim;
    device = dev;
    MCK(cudaSetDevice(device));
    const int np = n_params(in);
    MCK(cudaMalloc(&d_params, sizeof(float) * np * 4));  // params, grad, adam m, adam v
    d_grad = d_params + np;
    d_m = d_grad + np;
    d_v = d_m + np;
    MCK(cudaMemset(d_params, 0, sizeof(float) * np * 4));
    MCK(cudaMalloc(&d_scalar, sizeof(float) * 4));
    // He-uniform initialisation from a splitmix64 stream
    std::vector<float> h(np, 0.f);
    const Layout L = layout(in);
    uint64_t ctr = splitmix64(seed ^ 0x4d4c50ull);
    auto uni = [&](float lim) { return float((u01(splitmix64(ctr++)) * 2.0 - 1.0) * lim); };
    for (int i = 0; i < kH * in; ++i) h[L.w1 + i] = uni(std::sqrt(6.f / in));
    for (int i = 0; i < kH * kH; ++i) h[L.w2 + i] = uni(std::sqrt(6.f / kH));
    for (int i = 0; i < kH; ++i) h[L.w3 + i] = uni(std::sqrt(6.f / kH));
    MCK(cudaMemcpy(d_params, h.data(), sizeof(float) * np, cudaMemcpyHostToDevice));
    MCK(cudaFuncSetAttribute(k_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem_bytes(kMaxIn, true))));
    step = 0;
    return CUTS_OK;
}

void Mlp::destroy() {
    if (d_params) {
        cudaSetDevice(device);
        cudaFree(d_params);
        cudaFree(d_scalar);
        cudaFree(d_X);
    }
    d_params = d_grad = d_m = d_v = d_scalar = d_X = nullptr;
}

int Mlp::upload(const float *X, const float *T, int n) {
    if (n > cap_rows) {
        cudaFree(d_X);
        d_X = nullptr;
        cap_rows = 0;
        MCK(cudaMalloc(&d_X, sizeof(float) * size_t(n) * (in + 2)));
        cap_rows = n;
    }
    MCK(cudaMemcpy(d_X, X, sizeof(float) * size_t(n) * in, cudaMemcpyHostToDevice));
    if (T) MCK(cudaMemcpy(d_X + size_t(cap_rows) * in, T, sizeof(float) * n, cudaMemcpyHostToDevice));
    return CUTS_OK;
}

static int grid_for(int n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, std::min((n + kPerBlock - 1) / kPerBlock, sms * 2));
}

int Mlp::loss_grad(const float *X, const float *T, int n, float *loss, float *grad_out) {
    MCK(cudaSetDevice(device));
    int rc = upload(X, T, n);
    if (rc) return rc;
    const int np = n_params(in);
    MCK(cudaMemset(d_grad, 0, sizeof(float) * np));
    MCK(cudaMemset(d_scalar, 0, sizeof(float)));
    k_mlp<<<grid_for(n), kThreads, smem_bytes(in, true)>>>(d_params, in, d_X, d_X + size_t(cap_rows) * in,
                                                         n, nullptr, d_grad, d_scalar);
    MCK(cudaGetLastError());
    float l = 0;
    MCK(cudaMemcpy(&l, d_scalar, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l / float(std::max(n, 1));
    if (grad_out) MCK(cudaMemcpy(grad_out, d_grad, sizeof(float) * np, cudaMemcpyDeviceToHost));
    return CUTS_OK;
}

int Mlp::train(const float *X, const float *T, int n, int epochs, int batch, float lr,
               float *final_loss) {
    MCK(cudaSetDevice(device));
    int rc = upload(X, T, n);
    if (rc) return rc;
    const int np = n_params(in);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    if (batch <= 0 || batch > n) batch = n;
    const float *dT = d_X + size_t(cap_rows) * in;
    for (int e = 0; e < epochs; ++e) {
        for (int s0 = 0; s0 < n; s0 += batch) {
            const int nb = std::min(batch, n - s0);
            MCK(cudaMemsetAsync(d_grad, 0, sizeof(float) * np));
            k_mlp<<<grid_for(nb), kThreads, smem_bytes(in, true)>>>(d_params, in, d_X + size_t(s0) * in,
                                                                  dT + s0, nb, nullptr, d_grad, nullptr);
            ++step;
            const float c1 = 1.f - std::pow(b1, float(step)), c2 = 1.f - std::pow(b2, float(step));
            k_adam<<<(np + 255) / 256, 256>>>(d_params, d_grad, d_m, d_v, np, lr, b1, b2, eps, c1, c2);
        }
    }
    MCK(cudaGetLastError());
    if (final_loss) {
        MCK(cudaMemset(d_scalar, 0, sizeof(float)));
        k_mlp<<<grid_for(n), kThreads, smem_bytes(in, false)>>>(d_params, in, d_X, dT, n, nullptr, nullptr,
                                                              d_scalar);
        float l = 0;
        MCK(cudaMemcpy(&l, d_scalar, sizeof(float), cudaMemcpyDeviceToHost));
        *final_loss = l / float(std::max(n, 1));
    }
    MCK(cudaDeviceSynchronize());
    return CUTS_OK;
}

int Mlp::predict(const float *X, int n, float *Y) {
    MCK(cudaSetDevice(device));
    int rc = upload(X, nullptr, n);
    if (rc) return rc;
    float *dY = d_X + size_t(cap_rows) * in;  // reuse the target slot
    k_mlp<<<grid_for(n), kThreads, smem_bytes(in, false)>>>(d_params, in, d_X, nullptr, n, dY, nullptr,
                                                          nullptr);
    MCK(cudaGetLastError());
    MCK(cudaMemcpy(Y, dY, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return CUTS_OK;
}

int Mlp::get_params(float *out) {
    MCK(cudaSetDevice(device));
    MCK(cudaMemcpy(out, d_params, sizeof(float) * n_params(in), cudaMemcpyDeviceToHost));
    return CUTS_OK;
}

int Mlp::set_params(const float *p) {
    MCK(cudaSetDevice(device));
    MCK(cudaMemcpy(d_params, p, sizeof(float) * n_params(in), cudaMemcpyHostToDevice));
    const int np = n_params(in);
    MCK(cudaMemset(d_m, 0, sizeof(float) * np * 2));
    step = 0;
    return CUTS_OK;
}

}  // namespace cuts
