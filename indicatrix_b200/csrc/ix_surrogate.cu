// ix_surrogate.cu -- the learned surrogate's kernels: a BF16 GEMM on the tensor cores
// (mma.sync m16n8k16, FP32 accumulation) and the elementwise steps of an MLP's forward
// pass, MSE backward pass and Adam update, all on device pointers and the caller's
// stream (include/ix_surrogate.h).  The network maps stone design parameters to
// tilt-resolved brilliance / fire / scintillation; it is trained on metrics this library
// computes (ix_evaluate_gem_optical_metrics_batch) and screens candidate designs before
// the tracer re-evaluates the survivors.  No reference counterpart: the reference has no
// tracer-trained surrogate.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ix {
namespace mlp {
namespace {

constexpr int TM = 64, TN = 64, TK = 16;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// C[m x n] (row-major, ldc) = op(A) op(B), A and B bf16 row-major (lda, ldb); op(A) is
// m x k (A itself k x m when trans_a), op(B) is k x n (B itself n x k when trans_b).  A
// 64 x 64 tile per CTA, 4 warps of 16 rows x 64 columns (8 mma n-tiles each); the K loop
// stages 64 x 16 of op(A) and 16 x 64 of op(B) in shared memory, zero outside the matrix.
__global__ void __launch_bounds__(128) gemm_bf16_kernel(int trans_a, int trans_b, int m, int n, int k,
                                                        const __nv_bfloat16* __restrict__ a, int lda,
                                                        const __nv_bfloat16* __restrict__ b, int ldb,
                                                        float* __restrict__ c, int ldc) {
    __shared__ __nv_bfloat16 As[TM][TK + 8];
    __shared__ __nv_bfloat16 Bs[TK][TN + 8];
    const int row0 = blockIdx.y * TM, col0 = blockIdx.x * TN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    for (int k0 = 0; k0 < k; k0 += TK) {
        for (int e = threadIdx.x; e < TM * TK; e += blockDim.x) {
            const int r = e / TK, kk = e % TK;
            const int gr = row0 + r, gk = k0 + kk;
            __nv_bfloat16 v = zero;
            if (gr < m && gk < k) v = trans_a ? a[(size_t)gk * lda + gr] : a[(size_t)gr * lda + gk];
            As[r][kk] = v;
        }
        for (int e = threadIdx.x; e < TK * TN; e += blockDim.x) {
            const int kk = e / TN, cc = e % TN;
            const int gk = k0 + kk, gc = col0 + cc;
            __nv_bfloat16 v = zero;
            if (gk < k && gc < n) v = trans_b ? b[(size_t)gc * ldb + gk] : b[(size_t)gk * ldb + gc];
            Bs[kk][cc] = v;
        }
        __syncthreads();
        const int ar = warp * 16;
        const uint32_t a0 = pack2(As[ar + gid][2 * tig], As[ar + gid][2 * tig + 1]);
        const uint32_t a1 = pack2(As[ar + gid + 8][2 * tig], As[ar + gid + 8][2 * tig + 1]);
        const uint32_t a2 = pack2(As[ar + gid][2 * tig + 8], As[ar + gid][2 * tig + 9]);
        const uint32_t a3 = pack2(As[ar + gid + 8][2 * tig + 8], As[ar + gid + 8][2 * tig + 9]);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int nc = j * 8 + gid;
            const uint32_t b0 = pack2(Bs[2 * tig][nc], Bs[2 * tig + 1][nc]);
            const uint32_t b1 = pack2(Bs[2 * tig + 8][nc], Bs[2 * tig + 9][nc]);
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int cc = col0 + j * 8 + 2 * tig;
        const int r0 = row0 + warp * 16 + gid;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = r0 + 8 * h;
            if (r >= m) continue;
            if (cc < n) c[(size_t)r * ldc + cc] = acc[j][2 * h];
            if (cc + 1 < n) c[(size_t)r * ldc + cc + 1] = acc[j][2 * h + 1];
        }
    }
}

// z = x + bias[col]; h = relu(z) when relu, else z.  z kept in f32 (for the backward
// pass), h in f32 and bf16 (the next layer's input).
__global__ void bias_act_kernel(int m, int n, const float* __restrict__ x, const float* __restrict__ bias, int relu,
                                float* __restrict__ z, float* __restrict__ h, __nv_bfloat16* __restrict__ hb) {
    const int64_t total = (int64_t)m * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = x[i] + bias[i % n];
        const float o = relu ? fmaxf(v, 0.0f) : v;
        if (z) z[i] = v;
        if (h) h[i] = o;
        if (hb) hb[i] = __float2bfloat16_rn(o);
    }
}

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

// dz = dh * (z > 0) (f32 and bf16).
__global__ void relu_backward_kernel(int64_t total, const float* __restrict__ dh, const float* __restrict__ z,
                                     float* __restrict__ dz, __nv_bfloat16* __restrict__ dzb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const float g = z[i] > 0.0f ? dh[i] : 0.0f;
        dz[i] = g;
        dzb[i] = __float2bfloat16_rn(g);
    }
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

cudaError_t gemm_bf16(int trans_a, int trans_b, int m, int n, int k, const void* a, int lda, const void* b, int ldb,
                      float* c, int ldc, cudaStream_t s) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    const dim3 grid((n + TN - 1) / TN, (m + TM - 1) / TM);
    gemm_bf16_kernel<<<grid, 128, 0, s>>>(trans_a, trans_b, m, n, k, (const __nv_bfloat16*)a, lda,
                                          (const __nv_bfloat16*)b, ldb, c, ldc);
    return cudaGetLastError();
}
cudaError_t bias_act(int m, int n, const float* x, const float* bias, int relu, float* z, float* h, void* hb,
                     cudaStream_t s) {
    bias_act_kernel<<<grid_for((int64_t)m * n), 256, 0, s>>>(m, n, x, bias, relu, z, h, (__nv_bfloat16*)hb);
    return cudaGetLastError();
}
cudaError_t mse_grad(int m, int n, const float* y, const float* t, float* dy, void* dyb, float* loss,
                     cudaStream_t s) {
    mse_grad_kernel<<<grid_for((int64_t)m * n), 256, 0, s>>>(m, n, y, t, dy, (__nv_bfloat16*)dyb, loss);
    return cudaGetLastError();
}
cudaError_t relu_backward(int64_t total, const float* dh, const float* z, float* dz, void* dzb, cudaStream_t s) {
    relu_backward_kernel<<<grid_for(total), 256, 0, s>>>(total, dh, z, dz, (__nv_bfloat16*)dzb);
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

int ix_mlp_gemm_bf16(int trans_a, int trans_b, uint32_t m, uint32_t n, uint32_t k, const void* a, uint32_t lda,
                     const void* b, uint32_t ldb, float* c, uint32_t ldc, void* stream) {
    if (!a || !b || !c) return 1;
    return rc(ix::mlp::gemm_bf16(trans_a, trans_b, (int)m, (int)n, (int)k, a, (int)lda, b, (int)ldb, c, (int)ldc,
                                 st(stream)));
}
int ix_mlp_bias_act(uint32_t m, uint32_t n, const float* x, const float* bias, int relu, float* z, float* h,
                    void* hb, void* stream) {
    if (!x || !bias) return 1;
    return rc(ix::mlp::bias_act((int)m, (int)n, x, bias, relu, z, h, hb, st(stream)));
}
int ix_mlp_mse_grad(uint32_t m, uint32_t n, const float* y, const float* t, float* dy, void* dyb, float* loss,
                    void* stream) {
    if (!y || !t || !dy || !dyb) return 1;
    return rc(ix::mlp::mse_grad((int)m, (int)n, y, t, dy, dyb, loss, st(stream)));
}
int ix_mlp_relu_backward(uint64_t count, const float* dh, const float* z, float* dz, void* dzb, void* stream) {
    if (!dh || !z || !dz || !dzb) return 1;
    return rc(ix::mlp::relu_backward((int64_t)count, dh, z, dz, dzb, st(stream)));
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
