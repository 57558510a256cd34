/*
 * ix_surrogate.h -- the learned surrogate's device kernels: a BF16 tensor-core GEMM with
 * FP32 accumulation and the elementwise steps of an MLP's forward pass, MSE backward pass
 * and Adam update.  All pointers are device pointers; every call is enqueued on `stream`
 * (a cudaStream_t, NULL = the legacy default stream) and returns 0, or 1 on a launch
 * error.  bf16 buffers are 16-bit bfloat16 values; matrices are row-major.
 *
 * No reference counterpart: the reference's analytic metrics (color/metrics/) are what
 * the network learns to predict from a stone's design parameters, as a screen in front of
 * the tracer for design search (indicatrix_b200/surrogate.py).
 */
#ifndef IX_SURROGATE_H
#define IX_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[m x n] (ldc) = op(A) op(B); op(A) = A (m x k, lda) or A^T when trans_a (A is k x m);
 * op(B) = B (k x n, ldb) or B^T when trans_b (B is n x k). */
int ix_mlp_gemm_bf16(int trans_a, int trans_b, uint32_t m, uint32_t n, uint32_t k, const void* a, uint32_t lda,
                     const void* b, uint32_t ldb, float* c, uint32_t ldc, void* stream);
/* z = x + bias (per column); h = relu(z) or z; any of z, h (f32), hb (bf16) may be NULL. */
int ix_mlp_bias_act(uint32_t m, uint32_t n, const float* x, const float* bias, int relu, float* z, float* h,
                    void* hb, void* stream);
/* dy = 2 (y - t) / (m n) as f32 and bf16; *loss += mean squared error (loss may be NULL). */
int ix_mlp_mse_grad(uint32_t m, uint32_t n, const float* y, const float* t, float* dy, void* dyb, float* loss,
                    void* stream);
/* dz = dh where z > 0, else 0 (f32 and bf16). */
int ix_mlp_relu_backward(uint64_t count, const float* dh, const float* z, float* dz, void* dzb, void* stream);
/* db[c] = sum over the m rows of dz[r][c]. */
int ix_mlp_bias_grad(uint32_t m, uint32_t n, const float* dz, float* db, void* stream);
/* Adam step t (1-based) on f32 weights w with moments m, v; wb (bf16 copy) may be NULL. */
int ix_mlp_adam(uint64_t count, float* w, void* wb, const float* g, float* m, float* v, float lr, float beta1,
                float beta2, float eps, uint32_t t, void* stream);
/* xb = bf16(x). */
int ix_mlp_to_bf16(uint64_t count, const float* x, void* xb, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IX_SURROGATE_H */
