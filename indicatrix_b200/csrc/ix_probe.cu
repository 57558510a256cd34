// ix_probe.cu -- FP32 FMA-pipe throughput probe.
//
// The roofline denominator for the transport kernels, which are FP32-ALU bound: chains
// of independent fused multiply-adds, enough warps per SM to saturate the FMA pipe,
// timed with CUDA events.  Reported as FLOP/s counting an FMA as two operations.
#include <cuda_runtime.h>

#include <cstdint>

namespace ix {

constexpr int PROBE_ITERS = 8192;
constexpr int PROBE_CHAINS = 8;

__global__ void __launch_bounds__(256) fp32_probe_kernel(float* out, float a, float b) {
    float acc[PROBE_CHAINS];
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; ++c) acc[c] = (float)(threadIdx.x + c) * 1e-3f;
    for (int i = 0; i < PROBE_ITERS; ++i) {
#pragma unroll
        for (int c = 0; c < PROBE_CHAINS; ++c) acc[c] = fmaf(acc[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; ++c) s += acc[c];
    if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live, never true
}

// Runs the probe `reps` times on `stream`; returns the best FLOP/s in *flops.
cudaError_t fp32_probe(int sm_count, int reps, cudaStream_t stream, double* flops) {
    float* d_out = nullptr;
    cudaError_t e = cudaMalloc(&d_out, sizeof(float) * 4096);
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sm_count * 8, threads = 256;
    double best = 0.0;
    for (int r = 0; r < reps + 1; ++r) {
        cudaEventRecord(e0, stream);
        fp32_probe_kernel<<<blocks, threads, 0, stream>>>(d_out, 0.999999f, 1e-7f);
        cudaEventRecord(e1, stream);
        e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        double f = 2.0 * PROBE_CHAINS * (double)PROBE_ITERS * blocks * threads / (ms * 1e-3);
        if (r > 0 && f > best) best = f;  // first run is warm-up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    *flops = best;
    return e;
}

}  // namespace ix
