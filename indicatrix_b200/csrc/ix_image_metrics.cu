// ix_image_metrics.cu -- the image metrics of a batch of renders (include/ix_design.h): per
// view, brilliance (mean luminance), fire (luminance-weighted RMS chroma) and
// scintillation (spatial coefficient of variation of luminance) over the pixels whose
// primary ray enters the stone, from two half-sample renders of the view.  One CTA per
// view; f64 sums reduced in a fixed order, so a view's metrics do not depend on
// scheduling.
#include "ix_launch.h"

namespace ix {

namespace {

constexpr int THREADS = 256;

// Does the ray o + t dir (t > 0) enter the convex set {x : n_i . x + d_i <= 0}?  The slab
// bounds in f32; a ray parallel to a plane is inside it or misses the whole set.
__device__ bool ray_enters(const float4* __restrict__ planes, uint32_t n, float3 o, float3 dir) {
    float t_near = 0.0f, t_far = 3.0e38f;
    for (uint32_t i = 0; i < n; ++i) {
        const float4 p = planes[i];
        const float denom = p.x * dir.x + p.y * dir.y + p.z * dir.z;
        const float side = p.x * o.x + p.y * o.y + p.z * o.z + p.w;
        if (fabsf(denom) < 1e-12f) {
            if (side > 0.0f) return false;
            continue;
        }
        const float t = -side / denom;
        if (denom < 0.0f) t_near = fmaxf(t_near, t);
        else t_far = fminf(t_far, t);
        if (t_near > t_far) return false;
    }
    return true;
}

// Per view, jobs 2v and 2v + 1 are two renders of one scene over disjoint sample ranges
// (halves a and b, each as its per-sample mean).  With S = X + Y + Z, N = (X - S / 3,
// Y - S / 3) the pixel's chromaticity offset from the equal-energy white in unnormalised
// form, and Y the luminance of both halves together,
//   brilliance    = mean Y over the stone's pixels;
//   fire          = sqrt(sum N_a . N_b / sum S_a S_b): the RMS of the chromaticity offset
//                   |N| / S over the stone, each pixel weighted by S^2.  Products of
//                   independent halves have the noise-free |N|^2 and S^2 as expectations
//                   and no per-pixel ratio is formed, so per-pixel noise biases neither;
//   scintillation = sqrt(cov(Y_a, Y_b)) / mean Y: the spatial covariance of the halves,
//                   which per-pixel noise leaves unbiased, over the mean.
__global__ void __launch_bounds__(THREADS) image_metrics_kernel(const ix_scene* __restrict__ scenes,
                                                                const BatchJob* __restrict__ jobs,
                                                                const double* __restrict__ sums,
                                                                float* __restrict__ out) {
    const BatchJob ja = jobs[2 * (uint64_t)blockIdx.x], jb = jobs[2 * (uint64_t)blockIdx.x + 1];
    const ix_scene& sc = scenes[ja.scene];
    const ix_camera& c = sc.camera;
    const float w = (float)sc.width, h = (float)sc.height;
    const float aspect = w / h;
    const double inv_a = 1.0 / (double)ja.spp, inv_b = 1.0 / (double)jb.spp;
    const double inv_ab = 1.0 / ((double)ja.spp + (double)jb.spp);
    const double* pa = sums + ja.out_offset;
    const double* pb = sums + jb.out_offset;
    // count, sum Y, sum Ya, sum Yb, sum Ya Yb, sum N_a . N_b, sum S_a S_b
    double acc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < ja.n_pixels; i += THREADS) {
        const uint32_t y = i / sc.width, x = i - y * sc.width;
        // The pinhole ray through the pixel centre (the camera model of the transport).
        const float u = (((float)x + 0.5f) / w - 0.5f) * 2.0f * aspect * c.fov_tan;
        const float v = (0.5f - ((float)y + 0.5f) / h) * 2.0f * c.fov_tan;
        float3 d = make_float3(c.forward[0] + c.right[0] * u + c.up[0] * v, c.forward[1] + c.right[1] * u + c.up[1] * v,
                               c.forward[2] + c.right[2] * u + c.up[2] * v);
        const float inv = rsqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        d = make_float3(d.x * inv, d.y * inv, d.z * inv);
        const float3 o = make_float3(c.origin[0], c.origin[1], c.origin[2]);
        if (!ray_enters(reinterpret_cast<const float4*>(sc.planes), sc.n_planes, o, d)) continue;
        const uint64_t k = 3 * (uint64_t)i;
        const double Y = (pa[k + 1] + pb[k + 1]) * inv_ab;
        const double Xa = pa[k] * inv_a, Ya = pa[k + 1] * inv_a, Za = pa[k + 2] * inv_a;
        const double Xb = pb[k] * inv_b, Yb = pb[k + 1] * inv_b, Zb = pb[k + 2] * inv_b;
        const double sa = Xa + Ya + Za, sb = Xb + Yb + Zb;
        const double nxa = Xa - sa / 3.0, nya = Ya - sa / 3.0, nxb = Xb - sb / 3.0, nyb = Yb - sb / 3.0;
        acc[0] += 1.0;
        acc[1] += Y;
        acc[2] += Ya;
        acc[3] += Yb;
        acc[4] += Ya * Yb;
        acc[5] += nxa * nxb + nya * nyb;
        acc[6] += sa * sb;
    }
    // Fixed-order reduction: warps by shuffle, then one thread over the warps' partials.
    __shared__ double part[THREADS / 32][7];
    for (int q = 0; q < 7; ++q) {
        double val = acc[q];
        for (int off = 16; off > 0; off >>= 1) val += __shfl_down_sync(0xFFFFFFFFu, val, off);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5][q] = val;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int wi = 0; wi < THREADS / 32; ++wi)
            for (int q = 0; q < 7; ++q) t[q] += part[wi][q];
        float* o = out + 3 * (uint64_t)blockIdx.x;
        if (t[0] <= 0.0 || t[1] <= 0.0) {
            o[0] = o[1] = o[2] = 0.0f;
            return;
        }
        const double n = t[0], mean = t[1] / n;
        const double cov = t[4] / n - (t[2] / n) * (t[3] / n);
        o[0] = (float)mean;
        o[1] = t[6] > 0.0 ? (float)sqrt(fmax(t[5] / t[6], 0.0)) : 0.0f;
        o[2] = (float)(sqrt(fmax(cov, 0.0)) / mean);
    }
}

}  // namespace

cudaError_t launch_image_metrics(const ix_scene* scenes, const BatchJob* jobs, uint32_t n_views, const double* sums,
                                 float* out, cudaStream_t stream) {
    if (n_views == 0) return cudaSuccess;
    if (!scenes || !jobs || !sums || !out || n_views > 0x7FFFFFFFu) return cudaErrorInvalidValue;
    image_metrics_kernel<<<n_views, THREADS, 0, stream>>>(scenes, jobs, sums, out);
    return cudaGetLastError();
}

}  // namespace ix
