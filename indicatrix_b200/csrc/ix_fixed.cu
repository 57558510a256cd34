// ix_fixed.cu -- rounds the path-pool kernels' fixed-point per-pixel sums to f64.
//
// A pixel component's sum is held as three 64-bit words (t, a, b) worth
// t 2^24 + a 2^-16 + b 2^-56 (ix_launch.h, FIXED_WORDS).  The conversion carries b's and
// a's overflow past 40 bits upward, forms L = a 2^40 + b exactly in 128 bits and rounds it
// to f64 with a single rounding (its two 52-bit halves are exact doubles, so their one
// addition rounds the exact value), then adds t 2^24.  For t = 0 -- every sum below
// 2^24 -- the result is the exactly rounded sum of the samples.
#include "ix_launch.h"

namespace ix {

namespace {

__global__ void __launch_bounds__(256) fixed_to_f64_kernel(const unsigned long long* __restrict__ acc,
                                                         double* __restrict__ out, uint64_t n, int accumulate) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t p = i / 3, c = i - p * 3;
    const unsigned long long* w = acc + p * FIXED_WORDS + c * 3;
    const unsigned long long M40 = (1ull << 40) - 1ull;
    unsigned long long t = w[0], a = w[1], b = w[2];
    a += b >> 40;
    b &= M40;
    t += a >> 40;
    a &= M40;
    const unsigned __int128 L = ((unsigned __int128)a << 40) | b;  // < 2^80
    const unsigned long long hi = (unsigned long long)(L >> 52);
    const unsigned long long lo = (unsigned long long)(L & ((1ull << 52) - 1ull));
    const double frac = __dadd_rn(__ull2double_rn(hi) * 4503599627370496.0, __ull2double_rn(lo)) *
                        1.3877787807814457e-17;  // 2^52, 2^-56
    const double v = t ? __dadd_rn(__ull2double_rn(t) * 16777216.0, frac) : frac;
    out[i] = accumulate ? __dadd_rn(out[i], v) : v;
}

}  // namespace

cudaError_t launch_fixed_to_f64(const unsigned long long* acc, double* out, uint64_t n_pixels, int accumulate,
                                cudaStream_t stream) {
    if (n_pixels == 0) return cudaSuccess;
    if (!acc || !out) return cudaErrorInvalidValue;
    const uint64_t n = n_pixels * 3;
    const unsigned threads = 256;
    const uint64_t blocks = (n + threads - 1) / threads;
    if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    fixed_to_f64_kernel<<<(unsigned)blocks, threads, 0, stream>>>(acc, out, n, accumulate);
    return cudaGetLastError();
}

}  // namespace ix
