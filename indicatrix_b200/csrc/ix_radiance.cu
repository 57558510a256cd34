// ix_radiance.cu -- the kernels of the radiance codec's device forms (include/ix_radiance.h):
// per-pixel f64 sums -> the wire's f32 values, raw or byte-shuffled into 4 planes, and the
// decoder's unshuffle + valid-sample add (radiance/shuffle.rs:23-27, :128-150) into f32
// sums on the device.  Byte and integer work; the only arithmetic is the f64 -> f32
// rounding and one IEEE f32 add per component, as the host decoder does.
#include <cstdint>
#include <cuda_runtime.h>

namespace ix {
namespace rad {
namespace {

// Four values per thread: a plane's 4 bytes of them are one 32-bit store, so every plane
// is written with coalesced words.  `values` is a multiple of 3; the tail (< 4 values)
// goes byte by byte.
__global__ void __launch_bounds__(256) encode_kernel(const double* __restrict__ sums, uint64_t values, int shuffle,
                                                     uint8_t* __restrict__ out) {
    const uint64_t quads = values / 4;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < quads + 1;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = 4 * q;
        if (i0 >= values) break;
        const int cnt = (int)(values - i0 < 4 ? values - i0 : 4);
        uint32_t w[4] = {0, 0, 0, 0};
        for (int k = 0; k < cnt; ++k) w[k] = __float_as_uint(__double2float_rn(sums[i0 + k]));
        if (!shuffle) {
            uint32_t* o = reinterpret_cast<uint32_t*>(out);
            for (int k = 0; k < cnt; ++k) o[i0 + k] = w[k];
        } else if (cnt == 4) {
            for (int p = 0; p < 4; ++p) {
                const uint32_t sh = 8 * p;
                const uint32_t word = ((w[0] >> sh) & 0xFFu) | (((w[1] >> sh) & 0xFFu) << 8) |
                                      (((w[2] >> sh) & 0xFFu) << 16) | (((w[3] >> sh) & 0xFFu) << 24);
                // Plane p starts at p * values bytes: word-aligned only when values % 4 == 0.
                if ((values & 3) == 0)
                    reinterpret_cast<uint32_t*>(out + p * values)[q] = word;
                else
                    for (int k = 0; k < 4; ++k) out[p * values + i0 + k] = (uint8_t)(word >> (8 * k));
            }
        } else {
            for (int k = 0; k < cnt; ++k)
                for (int p = 0; p < 4; ++p) out[p * values + i0 + k] = (uint8_t)(w[k] >> (8 * p));
        }
    }
}

__device__ __forceinline__ float value_at(const uint8_t* __restrict__ b, uint64_t n, uint64_t i, int shuffled) {
    if (!shuffled) return __uint_as_float(reinterpret_cast<const uint32_t*>(b)[i]);
    return __uint_as_float((uint32_t)b[i] | ((uint32_t)b[n + i] << 8) | ((uint32_t)b[2 * n + i] << 16) |
                           ((uint32_t)b[3 * n + i] << 24));
}

__global__ void __launch_bounds__(256) decode_add_kernel(const uint8_t* __restrict__ payload, uint64_t pixels,
                                                         int shuffled, float* __restrict__ acc,
                                                         unsigned int* __restrict__ dropped) {
    const uint64_t n = 3 * pixels;
    unsigned int local = 0;
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < pixels;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const float x = value_at(payload, n, 3 * p, shuffled);
        const float y = value_at(payload, n, 3 * p + 1, shuffled);
        const float z = value_at(payload, n, 3 * p + 2, shuffled);
        if (isfinite(x) && isfinite(y) && isfinite(z) && x >= 0.0f && y >= 0.0f && z >= 0.0f) {
            acc[3 * p] = __fadd_rn(acc[3 * p], x);
            acc[3 * p + 1] = __fadd_rn(acc[3 * p + 1], y);
            acc[3 * p + 2] = __fadd_rn(acc[3 * p + 2], z);
        } else {
            ++local;
        }
    }
    // One atomic per warp.
    for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, off);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(dropped, local);
}

unsigned int blocks_for(uint64_t n) {
    const uint64_t b = (n + 255) / 256;
    return (unsigned int)(b < 1 ? 1 : (b > 148ull * 64 ? 148ull * 64 : b));
}

}  // namespace

cudaError_t launch_encode(const double* sums, uint64_t values, int shuffle, uint8_t* out, cudaStream_t s) {
    if (values == 0) return cudaSuccess;
    encode_kernel<<<blocks_for(values / 4 + 1), 256, 0, s>>>(sums, values, shuffle, out);
    return cudaGetLastError();
}

cudaError_t launch_decode_add(const uint8_t* payload, uint64_t pixels, int shuffled, float* acc,
                              unsigned int* dropped, cudaStream_t s) {
    if (pixels == 0) return cudaSuccess;
    decode_add_kernel<<<blocks_for(pixels), 256, 0, s>>>(payload, pixels, shuffled, acc, dropped);
    return cudaGetLastError();
}

}  // namespace rad
}  // namespace ix
