// Training kernels of the learned schedule cost model: a 3-layer MLP
// (in -> hidden -> hidden -> 1, ReLU, fp32) fit to log10 device times by mean
// squared error with Adam.  Parameters are one float array in the order of
// the model file (graphindor_b200/schedule_cost/train.py): W1 [hidden x in],
// b1 [hidden], W2 [hidden x hidden], b2 [hidden], w3 [hidden], b3 [1].
//
// Per step (a minibatch of B rows, gathered through an index array):
//   mlp_fwd_kernel     block per row, thread per hidden unit: h1, h2, y
//   mlp_bwd_kernel     block per row: dL/dy, dL/dh2 (pre-ReLU), dL/dh1
//   mlp_wgrad_kernel   thread per parameter: the sum over the batch's rows,
//                      in row order (deterministic)
//   mlp_adam_kernel    thread per parameter: Adam with decoupled weight
//                      decay on the weight matrices and w3, as the host trainer
// The host trainer (numpy) is the gradient oracle these kernels are checked
// against.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

struct MlpShape {
    int in, hidden;
    int64_t oW1, ob1, oW2, ob2, ow3, ob3, total;
};

MlpShape shape_of(int in, int hidden) {
    MlpShape s{in, hidden, 0, 0, 0, 0, 0, 0, 0};
    s.oW1 = 0;
    s.ob1 = s.oW1 + static_cast<int64_t>(hidden) * in;
    s.oW2 = s.ob1 + hidden;
    s.ob2 = s.oW2 + static_cast<int64_t>(hidden) * hidden;
    s.ow3 = s.ob2 + hidden;
    s.ob3 = s.ow3 + hidden;
    s.total = s.ob3 + 1;
    return s;
}

// Block r = batch row r (input row idx[r]); thread o = hidden unit o;
// blockDim.x == hidden.  Writes h1, h2 (post-ReLU) and y.
__global__ void mlp_fwd_kernel(MlpShape s, const float *__restrict__ P, const float *__restrict__ X,
                               const int32_t *__restrict__ idx, int rows, float *__restrict__ H1,
                               float *__restrict__ H2, float *__restrict__ Y) {
    extern __shared__ float sh[];  // hidden (h1) + hidden (h2 * w3)
    const int r = blockIdx.x, o = threadIdx.x, H = s.hidden, I = s.in;
    if (r >= rows || o >= H) return;  // the grid and block match exactly; kept as a guard
    const float *x = X + static_cast<int64_t>(idx[r]) * I;
    float a = P[s.ob1 + o];
    for (int j = 0; j < I; ++j) a += P[s.oW1 + static_cast<int64_t>(o) * I + j] * x[j];
    const float h1 = a > 0.f ? a : 0.f;
    H1[static_cast<int64_t>(r) * H + o] = h1;
    sh[o] = h1;
    __syncthreads();
    float b = P[s.ob2 + o];
    for (int i = 0; i < H; ++i) b += P[s.oW2 + static_cast<int64_t>(o) * H + i] * sh[i];
    const float h2 = b > 0.f ? b : 0.f;
    H2[static_cast<int64_t>(r) * H + o] = h2;
    sh[H + o] = h2 * P[s.ow3 + o];
    __syncthreads();
    if (o == 0) {
        float y = P[s.ob3];
        for (int i = 0; i < H; ++i) y += sh[H + i];
        Y[r] = y;
    }
}

// dL/dy = 2 (y - t) / B; G2 = dL/d(pre-ReLU of layer 2), G1 likewise for
// layer 1.  Block per row, thread per hidden unit.
__global__ void mlp_bwd_kernel(MlpShape s, const float *__restrict__ P, const float *__restrict__ T,
                               const int32_t *__restrict__ idx, int rows, const float *__restrict__ H1,
                               const float *__restrict__ H2, const float *__restrict__ Y, float *__restrict__ GY,
                               float *__restrict__ G1, float *__restrict__ G2) {
    extern __shared__ float g2s[];  // hidden
    const int r = blockIdx.x, o = threadIdx.x, H = s.hidden;
    if (r >= rows || o >= H) return;
    const float gy = 2.f * (Y[r] - T[idx[r]]) / static_cast<float>(rows);
    if (o == 0) GY[r] = gy;
    const float g2 = H2[static_cast<int64_t>(r) * H + o] > 0.f ? gy * P[s.ow3 + o] : 0.f;
    G2[static_cast<int64_t>(r) * H + o] = g2;
    g2s[o] = g2;
    __syncthreads();
    float g1 = 0.f;
    for (int k = 0; k < H; ++k) g1 += g2s[k] * P[s.oW2 + static_cast<int64_t>(k) * H + o];
    G1[static_cast<int64_t>(r) * H + o] = H1[static_cast<int64_t>(r) * H + o] > 0.f ? g1 : 0.f;
}

// Thread per parameter: the gradient summed over the batch rows in order.
__global__ void mlp_wgrad_kernel(MlpShape s, const float *__restrict__ X, const int32_t *__restrict__ idx, int rows,
                                 const float *__restrict__ H1, const float *__restrict__ H2,
                                 const float *__restrict__ GY, const float *__restrict__ G1,
                                 const float *__restrict__ G2, float *__restrict__ grad) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= s.total) return;
    const int H = s.hidden, I = s.in;
    float acc = 0.f;
    if (p < s.ob1) {  // W1[o][j]
        const int o = static_cast<int>(p / I), j = static_cast<int>(p % I);
        for (int r = 0; r < rows; ++r)
            acc += G1[static_cast<int64_t>(r) * H + o] * X[static_cast<int64_t>(idx[r]) * I + j];
    } else if (p < s.oW2) {  // b1[o]
        const int o = static_cast<int>(p - s.ob1);
        for (int r = 0; r < rows; ++r) acc += G1[static_cast<int64_t>(r) * H + o];
    } else if (p < s.ob2) {  // W2[o][i]
        const int64_t q = p - s.oW2;
        const int o = static_cast<int>(q / H), i = static_cast<int>(q % H);
        for (int r = 0; r < rows; ++r)
            acc += G2[static_cast<int64_t>(r) * H + o] * H1[static_cast<int64_t>(r) * H + i];
    } else if (p < s.ow3) {  // b2[o]
        const int o = static_cast<int>(p - s.ob2);
        for (int r = 0; r < rows; ++r) acc += G2[static_cast<int64_t>(r) * H + o];
    } else if (p < s.ob3) {  // w3[o]
        const int o = static_cast<int>(p - s.ow3);
        for (int r = 0; r < rows; ++r) acc += GY[r] * H2[static_cast<int64_t>(r) * H + o];
    } else {  // b3
        for (int r = 0; r < rows; ++r) acc += GY[r];
    }
    grad[p] = acc;
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the gradient plus wd * param for
// W1, W2 and w3, as the host trainer does.
__global__ void mlp_adam_kernel(MlpShape s, float *__restrict__ P, const float *__restrict__ grad,
                                float *__restrict__ M, float *__restrict__ V, float lr, float wd, float c1, float c2) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= s.total) return;
    const bool decay = p < s.ob1 || (p >= s.oW2 && p < s.ob2) || (p >= s.ow3 && p < s.ob3);
    const float g = grad[p] + (decay ? wd * P[p] : 0.f);
    const float m = 0.9f * M[p] + 0.1f * g;
    const float v = 0.999f * V[p] + 0.001f * g * g;
    M[p] = m;
    V[p] = v;
    P[p] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
}

struct Dev {
    std::vector<void *> ptrs;
    ~Dev() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T **p, size_t n) {
        cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

// One forward + backward over `rows` gathered rows; grad receives the
// parameter gradient of the mean squared error, loss (optional, host) the
// loss before the step.
cudaError_t step_grad(const MlpShape &s, const float *P, const float *X, const float *T, const int32_t *idx,
                      int rows, float *H1, float *H2, float *Y, float *GY, float *G1, float *G2, float *grad,
                      cudaStream_t st) {
    const size_t sh = 2 * sizeof(float) * s.hidden;
    mlp_fwd_kernel<<<rows, s.hidden, sh, st>>>(s, P, X, idx, rows, H1, H2, Y);
    mlp_bwd_kernel<<<rows, s.hidden, sh / 2, st>>>(s, P, T, idx, rows, H1, H2, Y, GY, G1, G2);
    const int64_t blocks = (s.total + 255) / 256;
    mlp_wgrad_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(s, X, idx, rows, H1, H2, GY, G1, G2, grad);
    return cudaGetLastError();
}

}  // namespace
}  // namespace gi

using namespace gi;

extern "C" {

int gi_mlp_grad(const float *X, const float *y, int rows, int in, int hidden, const float *params, float *grad_out,
                float *loss_out) {
    if (!X || !y || !params || !grad_out || rows < 1 || in < 1 || hidden < 1 || hidden > 1024)
        return fail(GI_EINVAL, "bad MLP arguments");
    const MlpShape s = shape_of(in, hidden);
    Dev d;
    float *dX, *dT, *dP, *H1, *H2, *Y, *GY, *G1, *G2, *dG;
    int32_t *dI;
    cudaError_t e;
    std::vector<int32_t> idx(rows);
    std::iota(idx.begin(), idx.end(), 0);
    if ((e = d.alloc(&dX, static_cast<size_t>(rows) * in)) != cudaSuccess || (e = d.alloc(&dT, rows)) != cudaSuccess ||
        (e = d.alloc(&dP, s.total)) != cudaSuccess || (e = d.alloc(&dI, rows)) != cudaSuccess ||
        (e = d.alloc(&H1, static_cast<size_t>(rows) * hidden)) != cudaSuccess ||
        (e = d.alloc(&H2, static_cast<size_t>(rows) * hidden)) != cudaSuccess || (e = d.alloc(&Y, rows)) != cudaSuccess ||
        (e = d.alloc(&GY, rows)) != cudaSuccess || (e = d.alloc(&G1, static_cast<size_t>(rows) * hidden)) != cudaSuccess ||
        (e = d.alloc(&G2, static_cast<size_t>(rows) * hidden)) != cudaSuccess || (e = d.alloc(&dG, s.total)) != cudaSuccess)
        return cuda_fail(e, "MLP allocation");
    if ((e = cudaMemcpy(dX, X, sizeof(float) * rows * in, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dT, y, sizeof(float) * rows, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dP, params, sizeof(float) * s.total, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dI, idx.data(), sizeof(int32_t) * rows, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "MLP upload");
    if ((e = step_grad(s, dP, dX, dT, dI, rows, H1, H2, Y, GY, G1, G2, dG, nullptr)) != cudaSuccess)
        return cuda_fail(e, "MLP kernels");
    std::vector<float> yh(rows);
    if ((e = cudaMemcpy(grad_out, dG, sizeof(float) * s.total, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(yh.data(), Y, sizeof(float) * rows, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "MLP download");
    if (loss_out) {
        double l = 0;
        for (int r = 0; r < rows; ++r) l += (yh[r] - y[r]) * static_cast<double>(yh[r] - y[r]);
        *loss_out = static_cast<float>(l / rows);
    }
    return GI_OK;
}

int gi_mlp_predict(const float *X, int rows, int in, int hidden, const float *params, float *y_out) {
    if (!X || !params || !y_out || rows < 1 || in < 1 || hidden < 1 || hidden > 1024)
        return fail(GI_EINVAL, "bad MLP arguments");
    const MlpShape s = shape_of(in, hidden);
    Dev d;
    float *dX, *dP, *H1, *H2, *Y;
    int32_t *dI;
    cudaError_t e;
    std::vector<int32_t> idx(rows);
    std::iota(idx.begin(), idx.end(), 0);
    if ((e = d.alloc(&dX, static_cast<size_t>(rows) * in)) != cudaSuccess || (e = d.alloc(&dP, s.total)) != cudaSuccess ||
        (e = d.alloc(&dI, rows)) != cudaSuccess || (e = d.alloc(&H1, static_cast<size_t>(rows) * hidden)) != cudaSuccess ||
        (e = d.alloc(&H2, static_cast<size_t>(rows) * hidden)) != cudaSuccess || (e = d.alloc(&Y, rows)) != cudaSuccess)
        return cuda_fail(e, "MLP allocation");
    if ((e = cudaMemcpy(dX, X, sizeof(float) * rows * in, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dP, params, sizeof(float) * s.total, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dI, idx.data(), sizeof(int32_t) * rows, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "MLP upload");
    mlp_fwd_kernel<<<rows, hidden, 2 * sizeof(float) * hidden>>>(s, dP, dX, dI, rows, H1, H2, Y);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpy(y_out, Y, sizeof(float) * rows, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "MLP forward");
    return GI_OK;
}

int gi_mlp_train(const float *X, const float *y, int rows, int in, int hidden, int epochs, int batch, float lr,
                 float wd, uint64_t seed, float *params_inout, float *loss_out) {
    if (!X || !y || !params_inout || rows < 1 || in < 1 || hidden < 1 || hidden > 1024 || epochs < 0 || batch < 1)
        return fail(GI_EINVAL, "bad MLP arguments");
    const MlpShape s = shape_of(in, hidden);
    const int B = std::min(batch, rows);
    Dev d;
    float *dX, *dT, *dP, *H1, *H2, *Y, *GY, *G1, *G2, *dG, *dM, *dV;
    int32_t *dI;
    cudaError_t e;
    const size_t maxr = static_cast<size_t>(rows);
    if ((e = d.alloc(&dX, maxr * in)) != cudaSuccess || (e = d.alloc(&dT, maxr)) != cudaSuccess ||
        (e = d.alloc(&dP, s.total)) != cudaSuccess || (e = d.alloc(&dI, maxr)) != cudaSuccess ||
        (e = d.alloc(&H1, maxr * hidden)) != cudaSuccess || (e = d.alloc(&H2, maxr * hidden)) != cudaSuccess ||
        (e = d.alloc(&Y, maxr)) != cudaSuccess || (e = d.alloc(&GY, maxr)) != cudaSuccess ||
        (e = d.alloc(&G1, maxr * hidden)) != cudaSuccess || (e = d.alloc(&G2, maxr * hidden)) != cudaSuccess ||
        (e = d.alloc(&dG, s.total)) != cudaSuccess || (e = d.alloc(&dM, s.total)) != cudaSuccess ||
        (e = d.alloc(&dV, s.total)) != cudaSuccess)
        return cuda_fail(e, "MLP allocation");
    if ((e = cudaMemcpy(dX, X, sizeof(float) * rows * in, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dT, y, sizeof(float) * rows, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dP, params_inout, sizeof(float) * s.total, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(dM, 0, sizeof(float) * s.total)) != cudaSuccess ||
        (e = cudaMemset(dV, 0, sizeof(float) * s.total)) != cudaSuccess)
        return cuda_fail(e, "MLP upload");
    // Minibatches of a seeded shuffle per epoch (splitmix64-driven
    // Fisher-Yates), uploaded as index arrays.
    std::vector<int32_t> order(rows);
    std::iota(order.begin(), order.end(), 0);
    uint64_t state = seed;
    auto next = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const int64_t blocks = (s.total + 255) / 256;
    int64_t t = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int i = rows - 1; i > 0; --i) std::swap(order[i], order[static_cast<int>(next() % (i + 1))]);
        if ((e = cudaMemcpy(dI, order.data(), sizeof(int32_t) * rows, cudaMemcpyHostToDevice)) != cudaSuccess)
            return cuda_fail(e, "MLP batch upload");
        for (int b0 = 0; b0 < rows; b0 += B) {
            const int nb = std::min(B, rows - b0);
            if ((e = step_grad(s, dP, dX, dT, dI + b0, nb, H1, H2, Y, GY, G1, G2, dG, nullptr)) != cudaSuccess)
                return cuda_fail(e, "MLP kernels");
            ++t;
            const float c1 = 1.f - std::pow(0.9f, static_cast<float>(t));
            const float c2 = 1.f - std::pow(0.999f, static_cast<float>(t));
            mlp_adam_kernel<<<static_cast<unsigned>(blocks), 256>>>(s, dP, dG, dM, dV, lr, wd, c1, c2);
            if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "MLP update");
        }
    }
    if ((e = cudaMemcpy(params_inout, dP, sizeof(float) * s.total, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "MLP download");
    if (loss_out) {
        std::vector<float> g(s.total);
        return gi_mlp_grad(X, y, rows, in, hidden, params_inout, g.data(), loss_out);
    }
    return GI_OK;
}

}  // extern "C"
