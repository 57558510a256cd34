// ix_kernels.cu -- the frame-tracing megakernel and the per-function check kernels.
//
// Compiled twice by the build (IX_EXACT=1 with -fmad=false, IX_EXACT=0 with
// contraction); every symbol is suffixed accordingly.
//
// Megakernel layout (GPU-first, not a translation of the reference's one-thread-per-tuple
// WGSL kernel):
//   * persistent CTAs; each CTA stages the stone's half-space planes (<= 128 x 16 B) in
//     shared memory once, and every slab scan reads them as warp-wide broadcasts;
//   * work is claimed a warp at a time from a global counter: one task is a run of
//     `pixels_per_task` consecutive pixels x all their samples, flattened pixel-major;
//     lane l takes flattened indices l, l+32, ... so a warp's 32 paths start in the same
//     pixel neighbourhood;
//   * a lane whose path finishes regenerates with its next sample while the other lanes
//     keep bouncing, so the bounce body (nearly all the arithmetic) stays converged
//     across lanes that are on different paths;
//   * per-pixel sums are accumulated in f64: each lane sums its own samples of a pixel
//     in ascending sample order into a shared-memory slot, then the warp folds the 32
//     slots in a fixed tree order.  The result depends only on (pixel, samples), never
//     on scheduling, so every run and every chunking of a frame gives the same bits.
#include "ix_launch.h"
#include "ix_transport.cuh"

#if IX_EXACT
#define IX_SFX(name) name##_exact
#else
#define IX_SFX(name) name##_fast
#endif

namespace ix {

constexpr int TRACE_MAX_PPT = 4;  // pixels per warp task held in the partial-sum table

__global__ void __launch_bounds__(128) IX_SFX(trace_kernel)(const __grid_constant__ TraceLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    extern __shared__ double s_part[];  // [warps][TRACE_MAX_PPT][32][3]
    const float4* gplanes = reinterpret_cast<const float4*>(L.scene.planes);
    for (uint32_t i = threadIdx.x; i < L.scene.n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    __syncthreads();

    const DevScene S{L.scene, L.absorbing};
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    double* part = s_part + (size_t)warp * TRACE_MAX_PPT * 32 * 3;
    const uint32_t ppt = L.pixels_per_task;
    const uint32_t spp = L.spp;
    const uint32_t n_tasks = (L.n_pixels + ppt - 1) / ppt;
    const uint32_t max_bounces = L.scene.max_bounces;
    unsigned long long drops = 0;

    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(L.task_counter, 1u);
        task = __shfl_sync(0xFFFFFFFFu, task, 0);
        if (task >= n_tasks) break;
        const uint32_t local0 = task * ppt;
        const uint32_t npix = min(ppt, L.n_pixels - local0);
        const uint32_t total = npix * spp;
        for (uint32_t j = 0; j < npix; ++j) {
            double* slot = part + ((size_t)j * 32 + lane) * 3;
            slot[0] = 0.0;
            slot[1] = 0.0;
            slot[2] = 0.0;
        }
        uint32_t q = lane;
        bool active = q < total;
        uint32_t cur_j = active ? q / spp : 0;
        double ax = 0.0, ay = 0.0, az = 0.0;
        PathState P;
        if (active) path_init(P, S, L.pixel_begin + local0 + cur_j, L.sample_offset + (q - cur_j * spp));
        while (__any_sync(0xFFFFFFFFu, active)) {
            if (!active) continue;
            float env[8];
            int r = (P.bounce >= max_bounces) ? (int)BOUNCE_KILLED : path_bounce(P, S, s_planes, env);
            if (r == BOUNCE_CONTINUE && P.bounce < max_bounces) continue;
            // The path finished (escaped, roulette, or reached the bounce cap).
            V3 xyz = path_finish(P, S, r == BOUNCE_ESCAPED, env);
            if (isfinite(xyz.x) && isfinite(xyz.y) && isfinite(xyz.z)) {
                ax += (double)xyz.x;
                ay += (double)xyz.y;
                az += (double)xyz.z;
            } else {
                ++drops;
            }
            q += 32;
            uint32_t j = (q < total) ? q / spp : 0xFFFFFFFFu;
            if (j != cur_j) {
                double* slot = part + ((size_t)cur_j * 32 + lane) * 3;
                slot[0] = ax;
                slot[1] = ay;
                slot[2] = az;
                ax = ay = az = 0.0;
                cur_j = j;
            }
            if (q < total)
                path_init(P, S, L.pixel_begin + local0 + cur_j, L.sample_offset + (q - cur_j * spp));
            else
                active = false;
        }
        __syncwarp();
        for (uint32_t j = 0; j < npix; ++j) {
            const double* slot = part + ((size_t)j * 32 + lane) * 3;
            double x = slot[0], y = slot[1], z = slot[2];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                x += __shfl_down_sync(0xFFFFFFFFu, x, off);
                y += __shfl_down_sync(0xFFFFFFFFu, y, off);
                z += __shfl_down_sync(0xFFFFFFFFu, z, off);
            }
            if (lane == 0) {
                double* o = L.out + (size_t)(local0 + j) * 3;
                if (L.accumulate) {
                    o[0] += x;
                    o[1] += y;
                    o[2] += z;
                } else {
                    o[0] = x;
                    o[1] = y;
                    o[2] = z;
                }
            }
        }
        __syncwarp();
    }
    if (drops && L.dropped) atomicAdd(L.dropped, drops);
}

// One reference function per thread, for the per-function parity checks.
__global__ void IX_SFX(check_kernel)(const __grid_constant__ CheckLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    const float4* gplanes = reinterpret_cast<const float4*>(L.scene.planes);
    for (uint32_t i = threadIdx.x; i < L.scene.n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    __syncthreads();
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= L.n) return;
    const DevScene S{L.scene, L.absorbing};
    const uint32_t* in = L.in + (size_t)row * L.in_stride;
    uint32_t* out = L.out + (size_t)row * L.out_stride;
    auto inf = [&](int i) { return __uint_as_float(in[i]); };
    auto put = [&](int i, float v) { out[i] = __float_as_uint(v); };
    switch (L.fn) {
        case CHECK_SAMPLE_DRAWS: {
            Draws d = sample_draws(in[0], in[1]);
            out[0] = d.seed;
            put(1, d.jx);
            put(2, d.jy);
            put(3, d.hero);
            break;
        }
        case CHECK_HERO_LAMBDAS: {
            float l[8];
            hero_wavelengths(inf(0), l);
            for (int k = 0; k < 8; ++k) put(k, l[k]);
            break;
        }
        case CHECK_DISPERSION: put(0, dispersion_eval(S.s.material.dispersion, inf(0))); break;
        case CHECK_CMF: {
            V3 c = cmf(inf(0));
            put(0, c.x);
            put(1, c.y);
            put(2, c.z);
            break;
        }
        case CHECK_D65: put(0, d65(inf(0))); break;
        case CHECK_EXP_LANE: put(0, exp_lane(inf(0))); break;
        case CHECK_TIR_DELTA: put(0, tir_phase_delta(inf(0), inf(1), inf(2))); break;
        case CHECK_FRESNEL: {
            float n1 = inf(0), n2 = inf(1), cos_i = inf(2);
            float eta = n1 / n2;
            float s2 = eta * eta * fmaf(cos_i, -cos_i, 1.0f);
            float cos_t = sqrtf(fmaxf(1.0f - s2, 0.0f));
            float rs, rp;
            fresnel_rs_rp(n1, n2, cos_i, cos_t, rs, rp);
            Stokes s = fresnel_reflect_apply(Stokes{inf(3), inf(4), inf(5), inf(6)}, rs, rp);
            put(0, s.i);
            put(1, s.q);
            put(2, s.u);
            put(3, s.v);
            put(4, rs);
            put(5, rp);
            break;
        }
        case CHECK_ENV: {
            const ix_environment& env = S.s.environment;
            Lighting Lg = direction_lighting(env, v3(inf(0), inf(1), inf(2)), v3(inf(4), inf(5), inf(6)));
            put(0, lighting_radiance(Lg, env, spectral_power(env, inf(3))));
            break;
        }
        case CHECK_INTERSECT: {
            Hit h = intersect_planes(s_planes, (int)S.s.n_planes, v3(inf(0), inf(1), inf(2)),
                                     v3(inf(3), inf(4), inf(5)));
            put(0, h.t);
            put(1, (float)h.facet);
            break;
        }
        case CHECK_TRACE:
        case CHECK_TRACE_RAY: {
            PathState P;
            if (L.fn == CHECK_TRACE)
                path_init(P, S, in[0], in[1]);
            else
                path_init_ray(P, S, Ray{v3(inf(0), inf(1), inf(2)), v3(inf(3), inf(4), inf(5))}, in[6],
                              inf(7));
            float env[8];
            int r = BOUNCE_CONTINUE;
            uint32_t iterations = 0;
            while (P.bounce < S.s.max_bounces) {
                r = path_bounce(P, S, s_planes, env);
                ++iterations;
                if (r != BOUNCE_CONTINUE) break;
            }
            V3 xyz = path_finish(P, S, r == BOUNCE_ESCAPED, env);
            put(0, xyz.x);
            put(1, xyz.y);
            put(2, xyz.z);
            out[3] = iterations;
            break;
        }
        case CHECK_CAMERA_RAY: {
            Draws d = sample_draws(in[0], in[1]);
            uint32_t x = in[0] % S.s.width, y = in[0] / S.s.width;
            Ray r = generate_ray(S.s.camera, (float)x, (float)y, (float)S.s.width, (float)S.s.height,
                                 d.jx, d.jy);
            put(0, r.origin.x);
            put(1, r.origin.y);
            put(2, r.origin.z);
            put(3, r.dir.x);
            put(4, r.dir.y);
            put(5, r.dir.z);
            break;
        }
        case CHECK_ABSORPTION: put(0, spectral_absorption(S.s.material.abs_o, inf(0))); break;
        default: break;
    }
}

static size_t trace_smem_bytes(int threads) {
    return (size_t)(threads / 32) * TRACE_MAX_PPT * 32 * 3 * sizeof(double);
}

cudaError_t IX_SFX(launch_trace)(const TraceLaunch& l, cudaStream_t stream) {
    if (l.pixels_per_task == 0 || l.pixels_per_task > (uint32_t)TRACE_MAX_PPT) return cudaErrorInvalidValue;
    if (l.threads % 32 != 0 || l.threads > 128 || l.threads <= 0) return cudaErrorInvalidValue;
    if (l.scene.n_planes > IX_MAX_PLANES) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(l.task_counter, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    IX_SFX(trace_kernel)<<<l.blocks, l.threads, trace_smem_bytes(l.threads), stream>>>(l);
    return cudaGetLastError();
}

cudaError_t IX_SFX(launch_check)(const CheckLaunch& l, cudaStream_t stream) {
    if (l.scene.n_planes > IX_MAX_PLANES) return cudaErrorInvalidValue;
    if (l.n == 0) return cudaSuccess;
    const int threads = 128;
    const int blocks = (int)((l.n + threads - 1) / threads);
    IX_SFX(check_kernel)<<<blocks, threads, 0, stream>>>(l);
    return cudaGetLastError();
}

int IX_SFX(trace_blocks_per_sm)(int threads, size_t* smem_bytes) {
    int blocks = 0;
    size_t smem = trace_smem_bytes(threads);
    if (smem_bytes) *smem_bytes = smem;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, IX_SFX(trace_kernel), threads, smem) != cudaSuccess)
        return 0;
    return blocks;
}

}  // namespace ix
