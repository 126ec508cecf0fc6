// Training kernels of the planner's cost model: a 3-layer MLP, FP32 throughout,
//     a1 = relu(W1 x + b1),  a2 = relu(W2 a1 + b2),  y = W3 a2 + b3,
// with a mean-squared-error loss against the measured log-times, its exact gradient, and an Adam step. Parameters
// are one flat array [W1 (H x D)][b1 (H)][W2 (H x H)][b2 (H)][W3 (H)][b3 (1)], row-major weights (out x in).
//
// Every reduction (the loss, each weight gradient) is a fixed-order sum: per-chunk partial sums over fixed row
// ranges, then the chunks in order. No floating-point atomics, so a training run is bit-reproducible on a device.
// The sizes are small (tens of thousands of rows, 64 units); the kernels favour that determinism over speed.

#include "kernels.hpp"

#include "../../include/crdfft.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

namespace crdfft
{
namespace mlp
{
namespace
{

constexpr int kChunks = 64; // row chunks of a gradient reduction
constexpr int kThreads = 256;

struct Layout
{
    int D, H;
    long long rows;
    const float* W1;
    const float* b1;
    const float* W2;
    const float* b2;
    const float* W3;
    const float* b3;
};

Layout layout(int D, int H, const float* p, long long rows)
{
    Layout l{D, H, rows, p, nullptr, nullptr, nullptr, nullptr, nullptr};
    l.b1 = l.W1 + static_cast<size_t>(H) * D;
    l.W2 = l.b1 + H;
    l.b2 = l.W2 + static_cast<size_t>(H) * H;
    l.W3 = l.b2 + H;
    l.b3 = l.W3 + H;
    return l;
}

// Z = X W^T + b (rows x N), A = relu(Z) when RELU (else A = Z). One thread per output element.
template <bool RELU>
__global__ void linear_fwd(const float* __restrict__ X, int K, const float* __restrict__ W, const float* __restrict__ b,
                           int N, long long rows, float* __restrict__ Z, float* __restrict__ A)
{
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= rows * N)
        return;
    const long long r = idx / N;
    const int o = static_cast<int>(idx - r * N);
    const float* x = X + r * K;
    const float* w = W + static_cast<long long>(o) * K;
    float s = b[o];
    for (int k = 0; k < K; ++k)
        s = fmaf(w[k], x[k], s);
    if (Z != nullptr)
        Z[idx] = s;
    A[idx] = RELU ? fmaxf(s, 0.0f) : s;
}

// dY = 2 (y - t) / rows, and per-block partial sums of (y - t)^2.
__global__ void loss_grad(const float* __restrict__ y, const float* __restrict__ t, long long rows,
                          float* __restrict__ dy, float* __restrict__ partial)
{
    __shared__ float red[kThreads];
    float acc = 0.0f;
    const float inv = 2.0f / static_cast<float>(rows);
    for (long long r = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; r < rows;
         r += static_cast<long long>(gridDim.x) * blockDim.x)
    {
        const float e = y[r] - t[r];
        dy[r] = inv * e;
        acc = fmaf(e, e, acc);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1)
    {
        if (threadIdx.x < s)
            red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        partial[blockIdx.x] = red[0];
}

__global__ void loss_final(const float* __restrict__ partial, int n, long long rows, float* __restrict__ loss)
{
    if (threadIdx.x == 0 && blockIdx.x == 0)
    {
        float s = 0.0f;
        for (int i = 0; i < n; ++i)
            s += partial[i];
        *loss = s / static_cast<float>(rows);
    }
}

// Partial weight/bias gradients of one layer over row chunk blockIdx.y: for output o = blockIdx.x,
// k < K: sum_r dZ[r][o] A[r][k], k == K: sum_r dZ[r][o].
__global__ void grad_w_partial(const float* __restrict__ dZ, const float* __restrict__ A, int N, int K,
                               long long rows, float* __restrict__ partial)
{
    const int o = blockIdx.x;
    const int chunk = blockIdx.y;
    const long long per = (rows + kChunks - 1) / kChunks;
    const long long r0 = chunk * per;
    const long long r1 = r0 + per < rows ? r0 + per : rows;
    for (int k = threadIdx.x; k <= K; k += blockDim.x)
    {
        float s = 0.0f;
        for (long long r = r0; r < r1; ++r)
        {
            const float g = dZ[r * N + o];
            s = fmaf(g, k < K ? A[r * K + k] : 1.0f, s);
        }
        partial[(static_cast<long long>(chunk) * N + o) * (K + 1) + k] = s;
    }
}

__global__ void grad_w_reduce(const float* __restrict__ partial, int N, int K, float* __restrict__ gW,
                              float* __restrict__ gb)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= N * (K + 1))
        return;
    float s = 0.0f;
    for (int c = 0; c < kChunks; ++c)
        s += partial[static_cast<long long>(c) * N * (K + 1) + idx];
    const int o = idx / (K + 1);
    const int k = idx - o * (K + 1);
    if (k < K)
        gW[o * K + k] = s;
    else
        gb[o] = s;
}

// dZprev[r][k] = (Zprev[r][k] > 0) * sum_o dZ[r][o] W[o][k]   (the ReLU derivative at the pre-activation)
__global__ void grad_in(const float* __restrict__ dZ, const float* __restrict__ W, const float* __restrict__ Zprev,
                        int N, int K, long long rows, float* __restrict__ dZprev)
{
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= rows * K)
        return;
    const long long r = idx / K;
    const int k = static_cast<int>(idx - r * K);
    float s = 0.0f;
    for (int o = 0; o < N; ++o)
        s = fmaf(dZ[r * N + o], W[static_cast<long long>(o) * K + k], s);
    dZprev[idx] = Zprev[idx] > 0.0f ? s : 0.0f;
}

__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, long long count, float lr, float b1, float b2, float eps, float c1,
                          float c2)
{
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

unsigned blocks(long long work) { return static_cast<unsigned>((work + kThreads - 1) / kThreads); }

// Workspace: Z1 A1 Z2 A2 (rows x H each), y dy (rows), dZ2 dZ1 (rows x H), partials, loss partials.
struct Ws
{
    float *Z1, *A1, *Z2, *A2, *y, *dy, *dZ2, *dZ1, *part, *lpart;
};

Ws carve(float* w, int D, int H, long long rows)
{
    Ws s{};
    s.Z1 = w;
    s.A1 = s.Z1 + rows * H;
    s.Z2 = s.A1 + rows * H;
    s.A2 = s.Z2 + rows * H;
    s.y = s.A2 + rows * H;
    s.dy = s.y + rows;
    s.dZ2 = s.dy + rows;
    s.dZ1 = s.dZ2 + rows * H;
    s.part = s.dZ1 + rows * H;
    s.lpart = s.part + static_cast<long long>(kChunks) * H * ((D > H ? D : H) + 1);
    return s;
}

constexpr int kLossBlocks = 128;

cudaError_t forward(const Layout& l, const float* x, float* y, const Ws& w, cudaStream_t st)
{
    linear_fwd<true><<<blocks(l.rows * l.H), kThreads, 0, st>>>(x, l.D, l.W1, l.b1, l.H, l.rows, w.Z1, w.A1);
    linear_fwd<true><<<blocks(l.rows * l.H), kThreads, 0, st>>>(w.A1, l.H, l.W2, l.b2, l.H, l.rows, w.Z2, w.A2);
    linear_fwd<false><<<blocks(l.rows), kThreads, 0, st>>>(w.A2, l.H, l.W3, l.b3, 1, l.rows, nullptr, y);
    return cudaGetLastError();
}

} // namespace
} // namespace mlp
} // namespace crdfft

using namespace crdfft::mlp;

extern "C" {

size_t crdfft_mlp_param_count(int32_t in_dim, int32_t hidden)
{
    if (in_dim < 1 || hidden < 1)
        return 0;
    return static_cast<size_t>(hidden) * in_dim + hidden + static_cast<size_t>(hidden) * hidden + hidden + hidden + 1;
}

size_t crdfft_mlp_workspace_floats(int32_t in_dim, int32_t hidden, int64_t rows)
{
    if (in_dim < 1 || hidden < 1 || rows < 1)
        return 0;
    const size_t r = static_cast<size_t>(rows), h = static_cast<size_t>(hidden);
    const size_t wide = static_cast<size_t>(in_dim > hidden ? in_dim : hidden) + 1;
    return 6 * r * h + 2 * r + static_cast<size_t>(kChunks) * h * wide + kLossBlocks;
}

crdfft_status crdfft_mlp_forward(int32_t in_dim, int32_t hidden, const float* params, const float* x, int64_t rows,
                                 float* y, float* workspace, void* stream)
{
    if (in_dim < 1 || hidden < 1 || rows < 1 || params == nullptr || x == nullptr || y == nullptr ||
        workspace == nullptr)
        return CRDFFT_INVALID_ARG;
    const Layout l = layout(in_dim, hidden, params, rows);
    const Ws w = carve(workspace, in_dim, hidden, rows);
    return forward(l, x, y, w, static_cast<cudaStream_t>(stream)) == cudaSuccess ? CRDFFT_OK : CRDFFT_LAUNCH;
}

crdfft_status crdfft_mlp_gradients(int32_t in_dim, int32_t hidden, const float* params, const float* x,
                                   const float* target, int64_t rows, float* grad, float* loss, float* workspace,
                                   void* stream)
{
    if (in_dim < 1 || hidden < 1 || rows < 1 || params == nullptr || x == nullptr || target == nullptr ||
        grad == nullptr || loss == nullptr || workspace == nullptr)
        return CRDFFT_INVALID_ARG;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Layout l = layout(in_dim, hidden, params, rows);
    const Ws w = carve(workspace, in_dim, hidden, rows);
    const int D = in_dim, H = hidden;
    float* gW1 = grad;
    float* gb1 = gW1 + static_cast<size_t>(H) * D;
    float* gW2 = gb1 + H;
    float* gb2 = gW2 + static_cast<size_t>(H) * H;
    float* gW3 = gb2 + H;
    float* gb3 = gW3 + H;
    if (forward(l, x, w.y, w, st) != cudaSuccess)
        return CRDFFT_LAUNCH;
    loss_grad<<<kLossBlocks, kThreads, 0, st>>>(w.y, target, rows, w.dy, w.lpart);
    loss_final<<<1, 32, 0, st>>>(w.lpart, kLossBlocks, rows, loss);
    // output layer (N = 1, K = H): dW3, db3; then dZ2 = relu'(Z2) * dy W3
    grad_w_partial<<<dim3(1, kChunks), kThreads, 0, st>>>(w.dy, w.A2, 1, H, rows, w.part);
    grad_w_reduce<<<blocks(H + 1), kThreads, 0, st>>>(w.part, 1, H, gW3, gb3);
    grad_in<<<blocks(rows * H), kThreads, 0, st>>>(w.dy, l.W3, w.Z2, 1, H, rows, w.dZ2);
    // layer 2 (N = H, K = H)
    grad_w_partial<<<dim3(H, kChunks), kThreads, 0, st>>>(w.dZ2, w.A1, H, H, rows, w.part);
    grad_w_reduce<<<blocks(static_cast<long long>(H) * (H + 1)), kThreads, 0, st>>>(w.part, H, H, gW2, gb2);
    grad_in<<<blocks(rows * H), kThreads, 0, st>>>(w.dZ2, l.W2, w.Z1, H, H, rows, w.dZ1);
    // layer 1 (N = H, K = D)
    grad_w_partial<<<dim3(H, kChunks), kThreads, 0, st>>>(w.dZ1, x, H, D, rows, w.part);
    grad_w_reduce<<<blocks(static_cast<long long>(H) * (D + 1)), kThreads, 0, st>>>(w.part, H, D, gW1, gb1);
    return cudaGetLastError() == cudaSuccess ? CRDFFT_OK : CRDFFT_LAUNCH;
}

crdfft_status crdfft_mlp_adam(float* params, const float* grad, float* m, float* v, int64_t count, int32_t step,
                              float lr, float beta1, float beta2, float eps, void* stream)
{
    if (params == nullptr || grad == nullptr || m == nullptr || v == nullptr || count < 1 || step < 1)
        return CRDFFT_INVALID_ARG;
    const float c1 = 1.0f - static_cast<float>(std::pow(static_cast<double>(beta1), step));
    const float c2 = 1.0f - static_cast<float>(std::pow(static_cast<double>(beta2), step));
    adam_step<<<blocks(count), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(params, grad, m, v, count, lr, beta1,
                                                                                  beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? CRDFFT_OK : CRDFFT_LAUNCH;
}

} // extern "C"
