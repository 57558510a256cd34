// ix_kernels.cu -- the frame-tracing megakernels and the per-function check kernels.
//
// Compiled twice by the build (IX_EXACT=1 with -fmad=false, IX_EXACT=0 with
// contraction); every symbol is suffixed accordingly.
//
// Megakernel layout (GPU-first; the reference's WGSL kernel runs one thread per
// (pixel, sample) tuple):
//   * a path is traced by an 8-lane group, one lane per hero-wavelength channel
//     (ix_transport.cuh); a warp holds 4 independent paths;
//   * persistent CTAs claim work a warp at a time from a global counter: one task is a
//     run of consecutive pixels x all their samples, flattened pixel-major; group gi of
//     the warp takes flattened paths gi, gi + 4, ...; a group whose path finishes starts
//     its next path while the other groups keep bouncing;
//   * the stone's half-space planes (<= 128 x 16 B) sit in shared memory and every slab
//     scan reads them as broadcasts;
//   * per-pixel sums are accumulated in f64, each group over its own samples of a pixel
//     in ascending order, then the 4 group partials are folded in a fixed order.  The
//     sums depend only on (pixel, samples), never on scheduling: every run and every
//     chunking of a frame gives the same bits.
// The batch kernel runs the same task loop over many scenes (stones x tilts) in one
// launch; each warp keeps the planes of the scene it is working on in its own
// shared-memory slot.
#include "ix_launch.h"
#include "ix_transport.cuh"

#if IX_EXACT
#define IX_SFX(name) name##_exact
#else
#define IX_SFX(name) name##_fast
#endif

namespace ix {

constexpr int TRACE_MAX_PPT = 8;     // pixels per warp task held in the partial-sum table
constexpr int GROUPS_PER_WARP = 4;   // paths in flight per warp (8 lanes each)
constexpr int WARPS_PER_CTA = 4;     // 128 threads

// Resident-CTA targets of the register variants 1 and 2.  The isotropic megakernel fits
// 6 or 8 CTAs per SM; the uniaxial one carries the per-lane 4x4 complex solves (about
// 200 registers unconstrained) and spills heavily below ~160, so its variants ask 3 or 4.
constexpr int UNI_MINB_1 = 3;
constexpr int UNI_MINB_2 = 4;

// A path's camera sample: its seed and hero draw and its camera ray.
struct PathSetup {
    uint32_t seed;
    float hero;
    float o[3], d[3];
};
// A warp's shared scratch: each group's f64 partial sums per task pixel, and each
// group's next PATH_PREP path setups.
constexpr int PATH_PREP = 8;
struct WarpScratch {
    double part[TRACE_MAX_PPT][GROUPS_PER_WARP][3];
    PathSetup setup[GROUPS_PER_WARP][PATH_PREP];
};

// What the attributed kernels record of a path (PathEvents, transport/path_events.rs:27),
// reduced to what classify_path reads: group-uniform bits plus the first exit direction.
enum : uint32_t {
    EV_FACET = 1u,      // a facet event happened (first_facet is Some)
    EV_ENTERED = 2u,    // ... and the first one left the ray inside the stone
    EV_EXITED = 4u,     // an inside-to-outside transition happened (first_exit is Some)
    EV_WINDOWED = 8u,   // ... through a facet whose outward normal has y < -0.05
    EV_ROULETTE = 16u,  // the loop stopped by Russian roulette
    EV_ESCAPED = 32u,   // the loop stopped because the ray met no facet
    EV_SCATTERED = 64u, // a Henyey-Greenstein scattering event happened
};

// Where a task's attribution records go: record (s, pixel0 + j) of the launch is at
// s * stride + pixel0 + j.
struct AttrTask {
    const ExitScorer* scorer;
    uint8_t* cls;
    float* y;
    uint32_t stride;  // the launch's pixel count
    uint32_t pixel0;  // the task's first pixel within the launch
};

// classify_path (color/metrics/attribution.rs:75-98) through class_index
// (renderer/attribution_map.rs:39-58).  A path that never exited is labelled by how it
// stopped (unexited_reason, attribution.rs:57): roulette, the bounce cap, or an escape.
IX_DEV uint32_t classify_path(uint32_t ev, V3 exit_dir, V3 observer, const ExitScorer& sc) {
    if (!(ev & EV_FACET)) return IX_CLASS_MISS;
    if (!(ev & EV_ENTERED)) return IX_CLASS_GLARE;
    if (!(ev & EV_EXITED)) {
        if (ev & EV_ROULETTE) return IX_CLASS_KILLED;
        return (ev & EV_ESCAPED) ? IX_CLASS_NO_INTERSECTION : IX_CLASS_BUDGET;
    }
    if (ev & EV_WINDOWED) return IX_CLASS_WINDOWED;
    if (exit_dir.y > 0.05f) {
        if (sc.shadowed(exit_dir, observer)) return IX_CLASS_SHADOW;
        return sc.lit(exit_dir) ? IX_CLASS_RETURNED : IX_CLASS_UNLIT;
    }
    return IX_CLASS_SIDE_EXIT;
}

// One warp task: pixels [pixel0, pixel0 + npix) x samples [sample_offset, +spp), written
// to out[0 .. 3 npix).  Returns the number of non-finite samples this lane dropped.
// UNI selects the transport instantiation (TransportClass);
// ATTR adds the event record of each path and writes its class and luminance to `at`
// (the traced arithmetic is the same: the record only reads the path state).
template <int UNI, bool ATTR = false>
IX_DEV uint32_t trace_task(const Group& g, const DevScene& S, const float4* __restrict__ planes,
                           uint32_t pixel0, uint32_t npix, uint32_t spp, uint32_t sample_offset,
                           WarpScratch& ws, double* out, int accumulate, const AttrTask* at = nullptr) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gi = lane >> 3;
    const uint32_t total = npix * spp;
    const uint32_t max_bounces = S.s.max_bounces;
    uint32_t drops = 0;  // non-finite samples this lane dropped
    auto& part = ws.part;
    PathSetup* const setup = ws.setup[gi];
    if (g.c == 0)
        for (uint32_t j = 0; j < npix; ++j) {
            part[j][gi][0] = 0.0;
            part[j][gi][1] = 0.0;
            part[j][gi][2] = 0.0;
        }
    uint32_t q = gi;
    uint32_t m = 0;  // the group's paths started so far: path m is q = gi + 4 m
    bool active = q < total;
    bool fresh = active;  // the group's next path still needs its setup
    uint32_t cur_j = active ? q / spp : 0;
    LanePath P;
    uint32_t ev = 0;  // ATTR: the path's event bits
    V3 exit_dir = v3(0.0f, 0.0f, 0.0f);
    while (__any_sync(0xFFFFFFFFu, active)) {
        if (!active) continue;
        // One setup site for the first path and every regenerated one keeps a single
        // copy of the setup code in the loop.
        if (fresh) {
            // Camera samples are prepared PATH_PREP paths at a time, lane c taking the
            // group's path m + c: one draw and camera ray per lane instead of the same
            // one on all 8 lanes.  The path then starts from its prepared slot.
            if (m % PATH_PREP == 0) {
                const uint32_t qc = gi + GROUPS_PER_WARP * (m + (uint32_t)g.c);
                if (qc < total) {
                    const uint32_t jc = qc / spp;
                    const uint32_t pixel = pixel0 + jc;
                    const Draws dr = sample_draws(pixel, sample_offset + (qc - jc * spp));
                    const ix_scene& sc = S.s;
                    const Ray r = generate_ray(sc.camera, (float)(pixel % sc.width), (float)(pixel / sc.width),
                                               (float)sc.width, (float)sc.height, dr.jx, dr.jy);
                    PathSetup& ps = setup[g.c];
                    ps.seed = dr.seed;
                    ps.hero = dr.hero;
                    ps.o[0] = r.origin.x, ps.o[1] = r.origin.y, ps.o[2] = r.origin.z;
                    ps.d[0] = r.dir.x, ps.d[1] = r.dir.y, ps.d[2] = r.dir.z;
                }
                __syncwarp(g.mask);
            }
            const PathSetup& ps = setup[m % PATH_PREP];
            const Ray r{v3(ps.o[0], ps.o[1], ps.o[2]), v3(ps.d[0], ps.d[1], ps.d[2])};
            group_init_ray<UNI>(g, P, S, r, ps.seed, ps.hero);
            ++m;
            fresh = false;
            ev = 0;
        }
        float esc = 0.0f;
        const bool capped = P.bounce >= max_bounces;
        const bool inside_before = P.inside;
        const int r = capped ? (int)BOUNCE_KILLED : group_step<UNI>(g, P, S, planes, esc);
        if constexpr (ATTR) {
            // A scattering step (the only step that leaves no plane of incidence behind)
            // records PathEvents::scatter (path_events.rs:96), no facet event; one ended by
            // its roulette is ScatterAbsorbed, which takes the roulette's class slot.
            const bool scatter_step = !capped && r != BOUNCE_ESCAPED && !P.has_prev;
            if (scatter_step) ev |= EV_SCATTERED;
            // record_facet (bounce_body.rs:680) runs after every facet dispatch, before
            // the roulette that may end the path; a miss records no facet event.
            if (!capped && r != BOUNCE_ESCAPED && !scatter_step) {
                if (!(ev & EV_FACET)) ev |= EV_FACET | (P.inside ? EV_ENTERED : 0u);
                if (inside_before && !P.inside && !(ev & EV_EXITED)) {
                    ev |= EV_EXITED | (planes[P.facet].y < -0.05f ? EV_WINDOWED : 0u);
                    exit_dir = P.d;
                }
            }
            if (r == BOUNCE_ESCAPED) ev |= EV_ESCAPED;
            if (r == BOUNCE_KILLED && !capped) ev |= EV_ROULETTE;
        }
        if (r == BOUNCE_CONTINUE && P.bounce < max_bounces) continue;
        // The path finished (escaped, roulette, or reached the bounce cap).
        const V3 xyz = group_finish<UNI>(g, P, S, r == BOUNCE_ESCAPED, esc);
        if constexpr (ATTR) {
            if (g.c == 0) {
                const size_t rec = (size_t)(q - cur_j * spp) * at->stride + at->pixel0 + cur_j;
                const uint32_t cls = classify_path(ev, exit_dir, P.observer, *at->scorer);
                // A hit's record carries the scattered flag in bit 6 (the classes are 0-8).
                at->cls[rec] = (uint8_t)(cls | ((cls != IX_CLASS_MISS && (ev & EV_SCATTERED)) ? 0x40u : 0u));
                at->y[rec] = xyz.y;
            }
        }
        // The group's f64 sums of this pixel live in its shared-memory slot (zeroed
        // above), added in the group's sample order.
        if (g.c == 0) {
            if (isfinite(xyz.x) && isfinite(xyz.y) && isfinite(xyz.z)) {
                part[cur_j][gi][0] += (double)xyz.x;
                part[cur_j][gi][1] += (double)xyz.y;
                part[cur_j][gi][2] += (double)xyz.z;
            } else {
                ++drops;
            }
        }
        q += GROUPS_PER_WARP;
        cur_j = (q < total) ? q / spp : 0;
        if (q < total)
            fresh = true;
        else
            active = false;
    }
    __syncwarp();
    // Fold each pixel's 4 group partials in a fixed order.
    if (lane < npix) {
        const uint32_t j = lane;
        double x = part[j][0][0], y = part[j][0][1], z = part[j][0][2];
#pragma unroll
        for (int k = 1; k < GROUPS_PER_WARP; ++k) {
            x += part[j][k][0];
            y += part[j][k][1];
            z += part[j][k][2];
        }
        double* o = out + (size_t)j * 3;
        if (accumulate) {
            o[0] += x;
            o[1] += y;
            o[2] += z;
        } else {
            o[0] = x;
            o[1] = y;
            o[2] = z;
        }
    }
    __syncwarp();
    return drops;
}

// Single scene: MINB is the resident CTAs per SM the register allocation must allow
// (1 = unconstrained).
template <int MINB, int UNI>
__global__ void __launch_bounds__(128, MINB) IX_SFX(trace_kernel)(const __grid_constant__ TraceLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    __shared__ WarpScratch s_scratch[WARPS_PER_CTA];
    const float4* gplanes = reinterpret_cast<const float4*>(L.scene.planes);
    for (uint32_t i = threadIdx.x; i < L.scene.n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    __syncthreads();
    const DevScene S = make_scene(L.scene, L.flags);
    const Group g = make_group();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ppt = L.pixels_per_task;
    const uint32_t n_tasks = (L.n_pixels + ppt - 1) / ppt;
    uint32_t drops = 0;  // non-finite samples this lane dropped
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(L.task_counter, 1u);
        task = __shfl_sync(0xFFFFFFFFu, task, 0);
        if (task >= n_tasks) break;
        const uint32_t local0 = task * ppt;
        const uint32_t npix = min(ppt, L.n_pixels - local0);
        drops += trace_task<UNI>(g, S, s_planes, L.pixel_begin + local0, npix, L.spp, L.sample_offset,
                                 s_scratch[threadIdx.x >> 5], L.out + (size_t)local0 * 3, L.accumulate);
    }
    if (drops && L.dropped) atomicAdd(L.dropped, (unsigned long long)drops);
}

// The trace kernel with spectral attribution: the same task loop, and each path's
// class code and luminance recorded for the fold.  Each CTA first derives the exit
// lighting's threshold (96 radiances and their median), which decides the classes.
template <int MINB, int UNI>
__global__ void __launch_bounds__(128, MINB)
    IX_SFX(trace_attributed_kernel)(const __grid_constant__ TraceLaunch L, const __grid_constant__ AttrLaunch A) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    __shared__ WarpScratch s_scratch[WARPS_PER_CTA];
    __shared__ float s_rad[96];
    __shared__ float s_threshold;
    const float4* gplanes = reinterpret_cast<const float4*>(L.scene.planes);
    for (uint32_t i = threadIdx.x; i < L.scene.n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    // Its barriers also publish the plane cache.
    const float threshold = exit_lighting_threshold<SCORE_ANY>(A.env, A.spec, A.factor, A.dirs, s_rad, &s_threshold);
    const ExitScorer scorer{A.env, A.spec, threshold, A.head_shadow_cos};
    const DevScene S = make_scene(L.scene, L.flags);
    const Group g = make_group();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ppt = L.pixels_per_task;
    const uint32_t n_tasks = (L.n_pixels + ppt - 1) / ppt;
    uint32_t drops = 0;  // non-finite samples this lane dropped
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) task = atomicAdd(L.task_counter, 1u);
        task = __shfl_sync(0xFFFFFFFFu, task, 0);
        if (task >= n_tasks) break;
        const uint32_t local0 = task * ppt;
        const uint32_t npix = min(ppt, L.n_pixels - local0);
        const AttrTask at{&scorer, A.cls, A.y, L.n_pixels, local0};
        drops += trace_task<UNI, true>(g, S, s_planes, L.pixel_begin + local0, npix, L.spp, L.sample_offset,
                                       s_scratch[threadIdx.x >> 5], L.out + (size_t)local0 * 3, L.accumulate, &at);
    }
    if (drops && L.dropped) atomicAdd(L.dropped, (unsigned long long)drops);
}

// AttributionPixel::add (renderer/attribution_map.rs:105-120), one thread per pixel, the
// launch's samples in ascending order: the f32 sums are formed exactly as the reference
// forms them (rounded adds and multiplies, no contraction), and the counts saturate.
__global__ void __launch_bounds__(128) IX_SFX(attribution_fold_kernel)(const __grid_constant__ AttrFoldLaunch L) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.n_pixels) return;
    ix_attribution_pixel a = L.map[p];
    auto sat = [](uint32_t v) { return v == 0xFFFFFFFFu ? v : v + 1u; };
    for (uint32_t s = 0; s < L.spp; ++s) {
        const size_t rec = (size_t)s * L.n_pixels + p;
        const uint32_t raw = L.cls[rec];
        const bool scattered = raw != IX_CLASS_MISS && (raw & 0x40u);
        const uint32_t c = raw == IX_CLASS_MISS ? raw : (raw & 0x3Fu);
        const float y = L.y[rec];
        a.samples = sat(a.samples);
        if (c >= IX_ATTRIBUTION_CLASSES) continue;
        a.hits = sat(a.hits);
        if (scattered) a.scattered = a.scattered + 1u;  // a plain add, as the reference's
        const bool finite = isfinite(y);
#pragma unroll
        for (uint32_t k = 0; k < IX_ATTRIBUTION_CLASSES; ++k) {
            if (k != c) continue;
            a.counts[k] = sat(a.counts[k]);
            if (finite) {
                a.y_sum[k] = __fadd_rn(a.y_sum[k], y);
                a.y_sq_sum[k] = __fadd_rn(a.y_sq_sum[k], __fmul_rn(y, y));
            }
        }
    }
    L.map[p] = a;
}

// Many scenes in one persistent launch (BatchLaunch): the task space is the
// concatenation of every job's tasks; a warp finds its job by binary search over the
// jobs' first-task offsets and reloads its plane slot only when the job's scene changes.
template <int MINB, int UNI>
__global__ void __launch_bounds__(128, MINB) IX_SFX(batch_kernel)(const __grid_constant__ BatchLaunch L) {
    __shared__ float4 s_planes[WARPS_PER_CTA][IX_MAX_PLANES];
    __shared__ WarpScratch s_scratch[WARPS_PER_CTA];
    const Group g = make_group();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    uint32_t cached = 0xFFFFFFFFu;
    uint32_t drops = 0;  // non-finite samples this lane dropped
    for (;;) {
        uint32_t claim = 0;
        if (lane == 0) claim = atomicAdd(L.task_counter, 1u);
        claim = __shfl_sync(0xFFFFFFFFu, claim, 0);
        const uint64_t task64 = (uint64_t)claim * L.stride;  // the claim's task
        if (task64 >= L.total_tasks) break;
        const uint32_t task = (uint32_t)task64;
        uint32_t lo = 0, hi = L.n_jobs;  // last job with task_begin <= task
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (L.jobs[mid].task_begin <= task)
                lo = mid;
            else
                hi = mid;
        }
        const BatchJob job = L.jobs[lo];
        const ix_scene& sc = L.scenes[job.scene];
        if (job.scene != cached) {
            __syncwarp();
            const float4* gp = reinterpret_cast<const float4*>(sc.planes);
            for (uint32_t i = lane; i < sc.n_planes; i += 32) s_planes[warp][i] = gp[i];
            __syncwarp();
            cached = job.scene;
        }
        const DevScene S = make_scene(sc, L.flags[job.scene]);
        const uint32_t local0 = (task - job.task_begin) * job.ppt;
        const uint32_t npix = min(job.ppt, job.n_pixels - local0);
        drops += trace_task<UNI>(g, S, s_planes[warp], local0, npix, job.spp, job.sample_offset, s_scratch[warp],
                                 L.out + job.out_offset + (size_t)local0 * 3, L.accumulate);
    }
    if (drops && L.dropped) atomicAdd(L.dropped, (unsigned long long)drops);
}

// Per-path checks: each 8-lane group traces one input row, exactly as the megakernel
// traces a path.
template <int UNI>
__global__ void __launch_bounds__(128) IX_SFX(check_trace_kernel)(const __grid_constant__ CheckLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    const float4* gplanes = reinterpret_cast<const float4*>(L.scene.planes);
    for (uint32_t i = threadIdx.x; i < L.scene.n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    __syncthreads();
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    if (row >= L.n) return;  // whole groups leave together (rows are group-aligned)
    const DevScene S = make_scene(L.scene, L.flags);
    const Group g = make_group();
    const uint32_t* in = L.in + (size_t)row * L.in_stride;
    uint32_t* out = L.out + (size_t)row * L.out_stride;
    LanePath P;
    if (L.fn == CHECK_TRACE) {
        group_init<UNI>(g, P, S, in[0], in[1]);
    } else {
        Ray r{v3(__uint_as_float(in[0]), __uint_as_float(in[1]), __uint_as_float(in[2])),
              v3(__uint_as_float(in[3]), __uint_as_float(in[4]), __uint_as_float(in[5]))};
        group_init_ray<UNI>(g, P, S, r, in[6], __uint_as_float(in[7]));
    }
    uint32_t it = 0;
    const V3 xyz = group_trace<UNI>(g, P, S, s_planes, &it);
    if (g.c == 0) {
        out[0] = __float_as_uint(xyz.x);
        out[1] = __float_as_uint(xyz.y);
        out[2] = __float_as_uint(xyz.z);
        out[3] = it;
    }
}

// One reference function per thread, for the per-function parity checks.
__global__ void IX_SFX(check_kernel)(const __grid_constant__ CheckLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    const float4* gplanes = reinterpret_cast<const float4*>(L.scene.planes);
    for (uint32_t i = threadIdx.x; i < L.scene.n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    __syncthreads();
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= L.n) return;
    const DevScene S = make_scene(L.scene, L.flags);
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
            put(0, environment_radiance_ext(S.s.environment, v3(inf(0), inf(1), inf(2)), v3(inf(4), inf(5), inf(6)),
                                            inf(3)));
            break;
        }
        case CHECK_INTERSECT: {
            Hit h = intersect_planes(s_planes, (int)S.s.n_planes, v3(inf(0), inf(1), inf(2)),
                                     v3(inf(3), inf(4), inf(5)));
            put(0, h.t);
            put(1, (float)h.facet);
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
        case CHECK_STOKES_ROTATE: {
            // The bounce's rotate_stokes_to_plane_of_incidence, as group_bounce calls it.
            Stokes st{inf(10), inf(11), inf(12), inf(13)};
            const V3 cpn = rotate_to_plane_of_incidence(st, in[9] != 0, v3(inf(6), inf(7), inf(8)),
                                                        v3(inf(0), inf(1), inf(2)), v3(inf(3), inf(4), inf(5)));
            put(0, st.i);
            put(1, st.q);
            put(2, st.u);
            put(3, st.v);
            put(4, cpn.x);
            put(5, cpn.y);
            put(6, cpn.z);
            break;
        }
        case CHECK_FRESNEL_CHANNEL: {
            // One channel of the bounce's reflect arm (the TIR retarder or the Fresnel
            // reflection, lane_scalar_reflect's arithmetic) and refract arm (the
            // transmission at the channel's own Snell angle), with the bounce's geometry.
            const float n1 = inf(0), n2 = inf(1), cos_i = inf(2);
            const Stokes st{inf(3), inf(4), inf(5), inf(6)};
            const float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
            const float sin_i = __fsqrt_rn(fmaxf(one_m_c2, 0.0f));
            const float ratio = __fdiv_rn(n1, n2);
            const float s2k = (ratio * ratio) * one_m_c2;
            for (int i = 0; i < 13; ++i) put(i, 0.0f);
            LanePath P;
            P.pdf = 1.0f;
            P.st = st;
            const Stokes r = lane_scalar_reflect(P, n1, n2, s2k, cos_i, sin_i);
            put(0, r.i);
            put(1, r.q);
            put(2, r.u);
            put(3, r.v);
            if (s2k > 1.0f) {
                put(12, 1.0f);
                break;
            }
            const float cos_t_k = __fsqrt_rn(fmaxf(1.0f - s2k, 0.0f));
            const float two = 2.0f * n1 * cos_i;
            const float t_s = two / fmaf(n2, cos_t_k, n1 * cos_i);
            const float t_p = two / fmaf(n1, cos_t_k, n2 * cos_i);
            const Stokes t = fresnel_transmit_apply(st, n1, n2, cos_i, cos_t_k, t_s, t_p);
            float rs, rp;
            fresnel_rs_rp(n1, n2, cos_i, cos_t_k, rs, rp);
            put(4, t.i);
            put(5, t.q);
            put(6, t.u);
            put(7, t.v);
            put(8, rs);
            put(9, rp);
            put(10, t_s);
            put(11, t_p);
            break;
        }
        case CHECK_CHANNEL_ALPHA: {
            const ix_material& m = S.s.material;
            put(0, iso_channel_alpha(m, spectral_absorption(m.abs_o, inf(3)), v3(inf(0), inf(1), inf(2))));
            break;
        }
        case CHECK_BIAXIAL: {
            const ix_material& m = S.s.material;
            const V3 k = v3(inf(0), inf(1), inf(2)), nn = v3(inf(3), inf(4), inf(5));
            const float cos_i = inf(6), lambda = inf(7), n_beta = inf(8);
            const BiaxFrame F = biax_frame(load3(m.c_axis));
            const Indicatrix I = make_indicatrix(m, n_beta);
            float ns, nf;
            wave_indices(I, F, k, ns, nf);
            put(0, ns);
            put(1, nf);
            auto put3 = [&](int i, V3 v) { put(i, v.x); put(i + 1, v.y); put(i + 2, v.z); };
            put3(2, eigen_polarization(I, F, k, true));
            put3(5, eigen_polarization(I, F, k, false));
            put3(8, mode_poynting_dir(I, F, k, true));
            put3(11, mode_poynting_dir(I, F, k, false));
            V3 d;
            put(14, resolve_entry_mode(I, F, k, nn, cos_i, n_beta, true, d));
            put3(15, d);
            put(18, resolve_entry_mode(I, F, k, nn, cos_i, n_beta, false, d));
            put3(19, d);
            const float ao = spectral_absorption(m.abs_o, lambda), ae = spectral_absorption(m.abs_e, lambda);
            const float ab = m.has_abs_beta ? spectral_absorption(m.abs_beta, lambda) : ao;
            put(22, biaxial_quadratic_form(F, ao, ab, ae, assigned_mode_e_field_biaxial(I, F, k, true)));
            put(23, biaxial_quadratic_form(F, ao, ab, ae, assigned_mode_e_field_biaxial(I, F, k, false)));
            break;
        }
        default: break;
    }
}

// The static task loop's kernels by (transport class, register budget): budgets 1 and 2
// are the occupancy targets of each transport (6 / 8 CTAs per SM isotropic, UNI_MINB_1 /
// UNI_MINB_2 for the uniaxial instantiations), 0 unconstrained.
template <int UNI>
struct TaskLoop {
    static constexpr int minb(int budget) {
        return budget == 1 ? (UNI ? UNI_MINB_1 : 6) : budget == 2 ? (UNI ? UNI_MINB_2 : 8) : 1;
    }
    using TraceFn = void (*)(const TraceLaunch);
    using BatchFn = void (*)(const BatchLaunch);
    static TraceFn trace(int budget) {
        switch (budget) {
            case 1: return IX_SFX(trace_kernel)<minb(1), UNI>;
            case 2: return IX_SFX(trace_kernel)<minb(2), UNI>;
            default: return IX_SFX(trace_kernel)<1, UNI>;
        }
    }
    static BatchFn batch(int budget) {
        switch (budget) {
            case 1: return IX_SFX(batch_kernel)<minb(1), UNI>;
            case 2: return IX_SFX(batch_kernel)<minb(2), UNI>;
            default: return IX_SFX(batch_kernel)<1, UNI>;
        }
    }
};
template <typename L>
static void start_task_loop(void (*kernel)(const L), const L& l, cudaStream_t stream) {
    kernel<<<l.blocks, l.threads, 0, stream>>>(l);
}

static bool launch_shape_ok(int threads) { return threads == 128; }

cudaError_t IX_SFX(launch_trace)(const TraceLaunch& l, cudaStream_t stream) {
    if (l.variant < 0 || l.variant >= N_VARIANTS) return cudaErrorInvalidValue;
    if (shape_is_pool(variant_shape(l.variant))) return IX_SFX(launch_pool_trace)(l, stream);
    if (l.pixels_per_task == 0 || l.pixels_per_task > (uint32_t)TRACE_MAX_PPT) return cudaErrorInvalidValue;
    if (!launch_shape_ok(l.threads)) return cudaErrorInvalidValue;
    if (l.scene.n_planes > IX_MAX_PLANES) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(l.task_counter, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    switch (transport_class(l.flags)) {
        case TRANSPORT_EXTENDED: start_task_loop(TaskLoop<TRANSPORT_EXTENDED>::trace(variant_budget(l.variant)), l, stream); break;
        case TRANSPORT_UNIAXIAL: start_task_loop(TaskLoop<TRANSPORT_UNIAXIAL>::trace(variant_budget(l.variant)), l, stream); break;
        default: start_task_loop(TaskLoop<TRANSPORT_ISOTROPIC>::trace(variant_budget(l.variant)), l, stream); break;
    }
    return cudaGetLastError();
}

// The attributed kernels carry one register budget each: the trace kernels' 6-CTA/SM
// variant (isotropic) and 3-CTA/SM variant (uniaxial).
constexpr int ATTR_MINB_ISO = 6;
constexpr int ATTR_MINB_UNI = UNI_MINB_1;

cudaError_t IX_SFX(launch_trace_attributed)(const TraceLaunch& l, const AttrLaunch& a, cudaStream_t stream) {
    if (l.pixels_per_task == 0 || l.pixels_per_task > (uint32_t)TRACE_MAX_PPT) return cudaErrorInvalidValue;
    if (!launch_shape_ok(l.threads)) return cudaErrorInvalidValue;
    if (l.scene.n_planes > IX_MAX_PLANES || !a.cls || !a.y) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(l.task_counter, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    switch (transport_class(l.flags)) {
        case TRANSPORT_EXTENDED:
            IX_SFX(trace_attributed_kernel)<ATTR_MINB_UNI, TRANSPORT_EXTENDED><<<l.blocks, l.threads, 0, stream>>>(l, a);
            break;
        case TRANSPORT_UNIAXIAL:
            IX_SFX(trace_attributed_kernel)<ATTR_MINB_UNI, TRANSPORT_UNIAXIAL><<<l.blocks, l.threads, 0, stream>>>(l, a);
            break;
        default:
            IX_SFX(trace_attributed_kernel)<ATTR_MINB_ISO, TRANSPORT_ISOTROPIC><<<l.blocks, l.threads, 0, stream>>>(l, a);
            break;
    }
    return cudaGetLastError();
}

cudaError_t IX_SFX(launch_attribution_fold)(const AttrFoldLaunch& l, cudaStream_t stream) {
    if (l.n_pixels == 0) return cudaSuccess;
    if (!l.cls || !l.y || !l.map) return cudaErrorInvalidValue;
    const int threads = 128;
    const int blocks = (int)((l.n_pixels + threads - 1) / threads);
    IX_SFX(attribution_fold_kernel)<<<blocks, threads, 0, stream>>>(l);
    return cudaGetLastError();
}

cudaError_t IX_SFX(launch_batch)(const BatchLaunch& l, cudaStream_t stream) {
    if (l.variant < 0 || l.variant >= N_VARIANTS) return cudaErrorInvalidValue;
    if (shape_is_pool(variant_shape(l.variant))) return IX_SFX(launch_pool_batch)(l, stream);
    if (!launch_shape_ok(l.threads) || l.n_jobs == 0 || l.stride == 0) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(l.task_counter, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    switch (l.uniaxial) {
        case TRANSPORT_EXTENDED: start_task_loop(TaskLoop<TRANSPORT_EXTENDED>::batch(variant_budget(l.variant)), l, stream); break;
        case TRANSPORT_UNIAXIAL: start_task_loop(TaskLoop<TRANSPORT_UNIAXIAL>::batch(variant_budget(l.variant)), l, stream); break;
        default: start_task_loop(TaskLoop<TRANSPORT_ISOTROPIC>::batch(variant_budget(l.variant)), l, stream); break;
    }
    return cudaGetLastError();
}

cudaError_t IX_SFX(launch_check)(const CheckLaunch& l, cudaStream_t stream) {
    if (l.scene.n_planes > IX_MAX_PLANES) return cudaErrorInvalidValue;
    if (l.n == 0) return cudaSuccess;
    const int threads = 128;
    if (l.fn == CHECK_TRACE || l.fn == CHECK_TRACE_RAY) {
        const int blocks = (int)((l.n * 8ull + threads - 1) / threads);
        switch (transport_class(l.flags)) {
            case TRANSPORT_EXTENDED: IX_SFX(check_trace_kernel)<TRANSPORT_EXTENDED><<<blocks, threads, 0, stream>>>(l); break;
            case TRANSPORT_UNIAXIAL: IX_SFX(check_trace_kernel)<TRANSPORT_UNIAXIAL><<<blocks, threads, 0, stream>>>(l); break;
            default: IX_SFX(check_trace_kernel)<TRANSPORT_ISOTROPIC><<<blocks, threads, 0, stream>>>(l); break;
        }
    } else {
        const int blocks = (int)((l.n + threads - 1) / threads);
        IX_SFX(check_kernel)<<<blocks, threads, 0, stream>>>(l);
    }
    return cudaGetLastError();
}

template <typename K>
static int occupancy(K kernel, int threads) {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, 0) != cudaSuccess) return 0;
    return blocks;
}

int IX_SFX(trace_blocks_per_sm)(int threads, int variant, int uniaxial, size_t* smem_bytes) {
    if (smem_bytes) *smem_bytes = 0;
    if (variant < 0 || variant >= N_VARIANTS) return 0;
    if (shape_is_pool(variant_shape(variant))) return IX_SFX(pool_trace_blocks_per_sm)(variant, uniaxial);
    if (threads != 128) return 0;
    const int budget = variant_budget(variant);
    switch (uniaxial) {
        case TRANSPORT_EXTENDED: return occupancy(TaskLoop<TRANSPORT_EXTENDED>::trace(budget), threads);
        case TRANSPORT_UNIAXIAL: return occupancy(TaskLoop<TRANSPORT_UNIAXIAL>::trace(budget), threads);
        default: return occupancy(TaskLoop<TRANSPORT_ISOTROPIC>::trace(budget), threads);
    }
}

int IX_SFX(trace_attributed_blocks_per_sm)(int threads, int uniaxial) {
    switch (uniaxial) {
        case TRANSPORT_EXTENDED: return occupancy(IX_SFX(trace_attributed_kernel)<ATTR_MINB_UNI, TRANSPORT_EXTENDED>, threads);
        case TRANSPORT_UNIAXIAL:
            return occupancy(IX_SFX(trace_attributed_kernel)<ATTR_MINB_UNI, TRANSPORT_UNIAXIAL>, threads);
        default: return occupancy(IX_SFX(trace_attributed_kernel)<ATTR_MINB_ISO, TRANSPORT_ISOTROPIC>, threads);
    }
}

int IX_SFX(batch_blocks_per_sm)(int threads, int variant, int uniaxial) {
    if (variant < 0 || variant >= N_VARIANTS) return 0;
    if (shape_is_pool(variant_shape(variant))) return IX_SFX(pool_batch_blocks_per_sm)(variant, uniaxial);
    if (threads != 128) return 0;
    const int budget = variant_budget(variant);
    switch (uniaxial) {
        case TRANSPORT_EXTENDED: return occupancy(TaskLoop<TRANSPORT_EXTENDED>::batch(budget), threads);
        case TRANSPORT_UNIAXIAL: return occupancy(TaskLoop<TRANSPORT_UNIAXIAL>::batch(budget), threads);
        default: return occupancy(TaskLoop<TRANSPORT_ISOTROPIC>::batch(budget), threads);
    }
}

}  // namespace ix
