// ix_surrogate.cu -- the learned surrogate's elementwise kernels: the MSE loss gradient,
// bias gradients, the Adam update and f32 -> bf16 conversion, all on device pointers and
// the caller's stream (include/ix_surrogate.h).  The GEMMs, with their bias / SiLU
// epilogues, are the tcgen05 kernels of ix_umma.cu.  The network maps stone design
// parameters to tilt-resolved brilliance / fire / scintillation measured on the tracer's
// renders (ix_design.h) and screens candidate designs before the tracer re-renders the
// survivors.  No reference counterpart: the reference has no tracer-trained surrogate.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ix {
namespace mlp {
namespace {

// Mean squared error over the m x n outputs: dy = 2 (y - t) / (m n) (f32 and bf16), and
// the loss summed into *loss (one atomic per warp).
__global__ void mse_grad_kernel(int m, int n, const float* __restrict__ y, const float* __restrict__ t,
                                float* __restrict__ dy, __nv_bfloat16* __restrict__ dyb, float* __restrict__ loss) {
    const int64_t total = (int64_t)m * n;
    const float inv = 1.0f / (float)total;
    float part = 0.0f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = y[i] - t[i];
        const float g = 2.0f * d * inv;
        dy[i] = g;
        dyb[i] = __float2bfloat16_rn(g);
        part += d * d * inv;
    }
    for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xFFFFFFFFu, part, off);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, part);
}

// db[col] = sum over rows of dz (one thread per column, rows in order).
__global__ void bias_grad_kernel(int m, int n, const float* __restrict__ dz, float* __restrict__ db) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= n) return;
    float s = 0.0f;
    for (int r = 0; r < m; ++r) s += dz[(size_t)r * n + col];
    db[col] = s;
}

// Adam on f32 master weights, with their bf16 copy refreshed (Kingma & Ba 2015).
__global__ void adam_kernel(int64_t count, float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                            const float* __restrict__ g, float* __restrict__ mom, float* __restrict__ vel, float lr,
                            float beta1, float beta2, float eps, float bias1, float bias2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = beta1 * mom[i] + (1.0f - beta1) * gi;
        const float vi = beta2 * vel[i] + (1.0f - beta2) * gi * gi;
        mom[i] = mi;
        vel[i] = vi;
        const float wi = w[i] - lr * (mi / bias1) / (sqrtf(vi / bias2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(int64_t count, const float* __restrict__ x, __nv_bfloat16* __restrict__ xb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        xb[i] = __float2bfloat16_rn(x[i]);
}

unsigned int grid_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (unsigned int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

cudaError_t mse_grad(int m, int n, const float* y, const float* t, float* dy, void* dyb, float* loss,
                     cudaStream_t s) {
    mse_grad_kernel<<<grid_for((int64_t)m * n), 256, 0, s>>>(m, n, y, t, dy, (__nv_bfloat16*)dyb, loss);
    return cudaGetLastError();
}
cudaError_t bias_grad(int m, int n, const float* dz, float* db, cudaStream_t s) {
    bias_grad_kernel<<<(n + 127) / 128, 128, 0, s>>>(m, n, dz, db);
    return cudaGetLastError();
}
cudaError_t adam(int64_t count, float* w, void* wb, const float* g, float* mom, float* vel, float lr, float beta1,
                 float beta2, float eps, float bias1, float bias2, cudaStream_t s) {
    adam_kernel<<<grid_for(count), 256, 0, s>>>(count, w, (__nv_bfloat16*)wb, g, mom, vel, lr, beta1, beta2, eps,
                                               bias1, bias2);
    return cudaGetLastError();
}
cudaError_t to_bf16(int64_t count, const float* x, void* xb, cudaStream_t s) {
    to_bf16_kernel<<<grid_for(count), 256, 0, s>>>(count, x, (__nv_bfloat16*)xb);
    return cudaGetLastError();
}

}  // namespace mlp
}  // namespace ix

#include "../../include/ix_surrogate.h"

#include <cmath>

namespace {
int rc(cudaError_t e) { return e == cudaSuccess ? 0 : 1; }
cudaStream_t st(void* s) { return (cudaStream_t)s; }
}  // namespace

extern "C" {

int ix_mlp_mse_grad(uint32_t m, uint32_t n, const float* y, const float* t, float* dy, void* dyb, float* loss,
                    void* stream) {
    if (!y || !t || !dy || !dyb) return 1;
    return rc(ix::mlp::mse_grad((int)m, (int)n, y, t, dy, dyb, loss, st(stream)));
}
int ix_mlp_bias_grad(uint32_t m, uint32_t n, const float* dz, float* db, void* stream) {
    if (!dz || !db) return 1;
    return rc(ix::mlp::bias_grad((int)m, (int)n, dz, db, st(stream)));
}
int ix_mlp_adam(uint64_t count, float* w, void* wb, const float* g, float* m, float* v, float lr, float beta1,
                float beta2, float eps, uint32_t t, void* stream) {
    if (!w || !g || !m || !v || t == 0) return 1;
    const float b1 = 1.0f - std::pow(beta1, (float)t), b2 = 1.0f - std::pow(beta2, (float)t);
    return rc(ix::mlp::adam((int64_t)count, w, wb, g, m, v, lr, beta1, beta2, eps, b1, b2, st(stream)));
}
int ix_mlp_to_bf16(uint64_t count, const float* x, void* xb, void* stream) {
    if (!x || !xb) return 1;
    return rc(ix::mlp::to_bf16((int64_t)count, x, xb, st(stream)));
}

}  // extern "C"
