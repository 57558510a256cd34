/*
 * ix_surrogate.h -- the learned surrogate's device kernels: BF16 GEMMs on the tcgen05
 * tensor cores with FP32 accumulation in tensor memory and fused epilogues (bias + SiLU
 * forward, SiLU derivative backward), and the elementwise steps of an MLP's MSE backward
 * pass and Adam update.  All pointers are device pointers; every call is enqueued on
 * `stream` (a cudaStream_t, NULL = the legacy default stream) and returns 0, or 1 on a
 * launch error or bad argument.  bf16 buffers hold 16-bit bfloat16 values; matrices are
 * row-major.
 *
 * No reference counterpart: the surrogate maps a stone's design parameters to the
 * brilliance / fire / scintillation the tracer measures on its renders
 * (ix_design.h), as a screen in front of the tracer for design search
 * (indicatrix_b200/surrogate.py).
 */
#ifndef IX_SURROGATE_H
#define IX_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[m x n] (ldc, f32) = op(A) op(B); op(A) = A (m x k, lda) or A^T when trans_a (A is
 * k x m); op(B) = B (k x n, ldb) or B^T when trans_b (B is n x k).  BF16 operands. */
int ix_mlp_gemm_bf16(int trans_a, int trans_b, uint32_t m, uint32_t n, uint32_t k, const void* a, uint32_t lda,
                     const void* b, uint32_t ldb, float* c, uint32_t ldc, void* stream);
/* One dense layer, y = x W^T + bias with x (m x k, ldx, bf16) and W (n x k, bf16): z = y
 * (f32, pre-activation), h = silu(y) when silu_act else y (f32), hb = bf16(h); any of z,
 * h, hb may be NULL; bias may be NULL (zero).  z, h, hb are m x n, row stride n. */
int ix_mlp_linear(uint32_t m, uint32_t n, uint32_t k, const void* x, uint32_t ldx, const void* w, const float* bias,
                  int silu_act, float* z, float* h, void* hb, void* stream);
/* Back through a layer and the previous SiLU: dz = (dz_next W) * silu'(z_prev), with
 * dz_next (m x k, bf16), W (k x n, bf16, the layer's weights), z_prev (m x n, f32); dz f32
 * and dzb bf16 (either may be NULL), m x n. */
int ix_mlp_backward_silu(uint32_t m, uint32_t n, uint32_t k, const void* dz_next, const void* w, const float* z_prev,
                         float* dz, void* dzb, void* stream);
/* Bit 0 set when a GEMM gave up waiting on its tensor-core completion barrier (its
 * output is then incomplete); reset clears it.  0xFFFFFFFF when it cannot be read. */
uint32_t ix_mlp_status(int reset);
/* dy = 2 (y - t) / (m n) as f32 and bf16; *loss += mean squared error (loss may be NULL). */
int ix_mlp_mse_grad(uint32_t m, uint32_t n, const float* y, const float* t, float* dy, void* dyb, float* loss,
                    void* stream);
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
