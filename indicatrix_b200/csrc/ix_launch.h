// ix_launch.h -- internal interface between the C-ABI host code (ix_backend.cpp) and the
// kernel translation unit, which is compiled twice (reference-exact rounding and fused
// rounding).  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ix_attribution.h"
#include "../../include/ix_cuda.h"
#include "../../include/ix_scene.h"

namespace ix {

// Per-scene transport flags, resolved on the host from the material.
enum : uint32_t {
    SCENE_ABSORBING = 1u,   // the o-ray or e-ray absorption has a non-zero term
    SCENE_UNIAXIAL = 2u,    // uniaxial birefringence (ix_material::anisotropic)
    SCENE_PLEOCHROIC = 4u,  // the o-ray and e-ray absorption differ
    SCENE_SCATTERING = 8u,  // Henyey-Greenstein interior scattering (scattering_sigma_s > 0)
    SCENE_ROUNDED = 16u,    // rounded facet edges (edge_rounding_radius > 0)
    SCENE_BIAXIAL = 32u,    // biaxial indicatrix (ix_material::biaxial, with anisotropic)
    SCENE_CONCAVE = 64u,    // concave tools carved out of the stone (ix_scene::n_tools > 0)
    SCENE_ENV_EXTENDED = 128u,  // a lighting model past the studio rig and iso-hemisphere
};
inline bool absorption_present(const ix_absorption& a) {
    if (a.has_spline) return true;
    for (uint32_t i = 0; i < a.n_bands && i < IX_MAX_BANDS; ++i)
        if (a.bands[i].peak != 0.0f) return true;
    return false;
}
inline bool absorption_equal(const ix_absorption& a, const ix_absorption& b) {
    if (a.n_bands != b.n_bands || a.has_spline != b.has_spline) return false;
    for (uint32_t i = 0; i < a.n_bands && i < IX_MAX_BANDS; ++i) {
        const ix_band &x = a.bands[i], &y = b.bands[i];
        if (x.center_nm != y.center_nm || x.width_nm != y.width_nm || x.peak != y.peak || x.shape != y.shape)
            return false;
    }
    if (a.has_spline)
        for (int i = 0; i < IX_SPLINE_KNOTS; ++i)
            if (a.spline[i] != b.spline[i]) return false;
    return true;
}
inline uint32_t scene_flags(const ix_material& m) {
    uint32_t f = 0;
    if (absorption_present(m.abs_o) || absorption_present(m.abs_e)) f |= SCENE_ABSORBING;
    if (m.biaxial && m.has_abs_beta && absorption_present(m.abs_beta)) f |= SCENE_ABSORBING;
    if (m.anisotropic) f |= SCENE_UNIAXIAL;
    if (m.anisotropic && m.biaxial) f |= SCENE_BIAXIAL;
    if (!absorption_equal(m.abs_o, m.abs_e)) f |= SCENE_PLEOCHROIC;
    if (m.scattering_sigma_s > 0.0f) f |= SCENE_SCATTERING;
    if (m.edge_rounding_radius > 0.0f) f |= SCENE_ROUNDED;
    return f;
}
// The isotropic megakernel assumes equal o/e absorption and no birefringence; any other
// scene runs the uniaxial instantiation of the transport.
inline bool needs_uniaxial_kernel(uint32_t flags) {
    return (flags & (SCENE_UNIAXIAL | SCENE_PLEOCHROIC | SCENE_SCATTERING | SCENE_ROUNDED | SCENE_BIAXIAL |
                     SCENE_CONCAVE | SCENE_ENV_EXTENDED)) != 0;
}
// The scene's flags: its material's, and whether tools carve it.
inline uint32_t scene_flags(const ix_scene& s) {
    const uint32_t m = s.environment.model;
    const bool env_ext = (m != IX_ENV_STUDIO && m != IX_ENV_ISO_HEMISPHERE && m != IX_ENV_UNIFORM) ||
                         s.environment.spectrum > IX_SPEC_FLAT;
    return scene_flags(s.material) | (s.n_tools ? SCENE_CONCAVE : 0u) | (env_ext ? SCENE_ENV_EXTENDED : 0u);
}
// The transport instantiation a scene needs: the isotropic megakernel, the uniaxial one,
// or the extended one -- the uniaxial bounce plus the out-of-line biaxial bounce, the
// carved-stone intersection and every lighting model -- which serves every scene, so a
// batch takes the largest of its scenes' classes.
enum TransportClass : int { TRANSPORT_ISOTROPIC = 0, TRANSPORT_UNIAXIAL = 1, TRANSPORT_EXTENDED = 2 };
constexpr int N_TRANSPORT_CLASSES = 3;
inline int transport_class(uint32_t flags) {
    if (flags & (SCENE_BIAXIAL | SCENE_CONCAVE | SCENE_ENV_EXTENDED)) return TRANSPORT_EXTENDED;
    return needs_uniaxial_kernel(flags) ? TRANSPORT_UNIAXIAL : TRANSPORT_ISOTROPIC;
}

// Launch shapes of the trace megakernels.  A shape is a task loop and a CTA size:
//  * SHAPE_TASKS: the static task loop (a warp task is a run of whole pixels x all their
//    samples, its paths split over the 4 groups of the warp by a fixed stride; per-pixel
//    f64 sums folded in a fixed order), 128 threads;
//  * SHAPE_POOL_*: the path-pool loop (a warp claims 32 paths at a time, prepares their
//    camera samples one per lane, and each 8-lane group takes the next prepared path
//    whenever its own finishes; samples are added into per-pixel fixed-point sums, which
//    no order of arrival changes), 128, 64 or 256 threads.
// A kernel variant is budget + 3 * shape, the budget being the register allocation's
// resident-warp target (0 unconstrained, 1 and 2 the two occupancy targets of each loop).
enum LaunchShape : int { SHAPE_TASKS = 0, SHAPE_POOL_128 = 1, SHAPE_POOL_64 = 2, SHAPE_POOL_256 = 3 };
constexpr int N_SHAPES = 4;
constexpr int N_BUDGETS = 3;
constexpr int N_VARIANTS = N_SHAPES * N_BUDGETS;
inline int variant_shape(int v) { return v / N_BUDGETS; }
inline int variant_budget(int v) { return v % N_BUDGETS; }
inline int shape_threads(int shape) { return shape == SHAPE_POOL_64 ? 64 : shape == SHAPE_POOL_256 ? 256 : 128; }
inline bool shape_is_pool(int shape) { return shape != SHAPE_TASKS; }

// Fixed-point per-pixel sums of the path-pool kernels: for each of X, Y and Z three 64-bit
// words (t, a, b) holding t 2^24 + a 2^-16 + b 2^-56.  A sample adds its exact binary
// expansion split into those digits (a and b below 2^40, so no word carries within a
// launch of up to FIXED_MAX_SAMPLES samples per pixel); the sum is exact, whatever the
// order the samples arrive in, and is rounded to f64 once by the conversion kernel.
constexpr int FIXED_WORDS = 9;
constexpr uint32_t FIXED_MAX_SAMPLES = 1u << 22;  // samples of one pixel in one launch
constexpr float FIXED_MAX_VALUE = 4.611686018427387904e18f;  // 2^62: larger samples are dropped

// One frame-tracing launch over the pixels [pixel_begin, pixel_begin + n_pixels).
struct TraceLaunch {
    ix_scene scene;            // `planes` is a device pointer here
    uint32_t flags;            // scene_flags(scene)
    uint32_t pixel_begin;
    uint32_t n_pixels;
    uint32_t sample_offset;
    uint32_t spp;
    uint32_t pixels_per_task;  // consecutive pixels one warp task covers (SHAPE_TASKS)
    double* out;               // device, n_pixels * 3 per-pixel sums
    int accumulate;            // 1: out += sums, 0: out = sums
    uint32_t* task_counter;    // device, zeroed by the launcher
    unsigned long long* dropped;  // device, non-finite samples dropped (may be null)
    unsigned long long* acc;   // device, n_pixels * FIXED_WORDS fixed-point sums (pool shapes)
    int blocks;                // persistent grid size
    int threads;               // threads per block (multiple of 32)
    int variant;               // budget + 3 * shape (see LaunchShape)
};

// One job of a batched launch: `n_pixels` pixels of scene `scene` x `spp` samples from
// `sample_offset`; the static task loop splits it into tasks of `ppt` pixels starting at
// global task `task_begin`, the path-pool loop into chunks of 32 paths (sample-major:
// path i is sample i / n_pixels of pixel i % n_pixels) starting at global chunk
// `chunk_begin`.  Its per-pixel sums go to out + out_offset (3 doubles per pixel) and,
// for the path-pool loop, its fixed-point sums to acc + acc_offset (FIXED_WORDS per pixel).
struct BatchJob {
    uint32_t scene;
    uint32_t n_pixels;
    uint32_t spp;
    uint32_t ppt;
    uint32_t task_begin;
    uint32_t sample_offset;
    uint64_t out_offset;
    uint32_t chunk_begin;
    uint32_t paths;
    uint64_t acc_offset;
};

struct BatchLaunch {
    const ix_scene* scenes;      // device array; each scene's `planes` is a device pointer
    const uint32_t* flags;       // device, scene_flags per scene
    uint32_t uniaxial;           // the plan's transport class (TransportClass): the largest of its scenes'
    const BatchJob* jobs;        // device, ascending task_begin and chunk_begin
    uint32_t n_jobs;
    uint32_t total_tasks;
    uint32_t total_chunks;
    double* out;
    int accumulate;
    uint32_t* task_counter;
    unsigned long long* dropped;
    unsigned long long* acc;     // device, FIXED_WORDS per pixel of every job (pool shapes)
    uint32_t stride;             // the k-th claim takes task / chunk k * stride (1: all of them;
                                 // the autotuner times variants on a strided sample)
    int blocks;
    int threads;
    int variant;                 // budget + 3 * shape
};

// The wavefront pipeline over a batch plan of isotropic scenes (ix_wavefront.cu): path
// slots whose state lives in HBM (one record per slot: path words once per path, lane
// words per channel), six
// queues of `capacity` slot indices and their counts, and the claim counter over the
// plan's padded path space (each job's paths start at 32 x its chunk_begin).
enum : int { WF_ACTIVE0 = 0, WF_ACTIVE1 = 1, WF_REFLECT = 2, WF_REFRACT = 3, WF_FROSTED = 4, WF_FINISH = 5,
             WF_QUEUES = 6 };
constexpr int VARIANT_WAVEFRONT = N_VARIANTS;  // the batch plans' variant id of the wavefront
struct WaveLaunch {
    const ix_scene* scenes;
    const uint32_t* flags;
    const BatchJob* jobs;
    uint32_t n_jobs;
    unsigned long long total_slots;  // 32 x the plan's chunks
    unsigned long long* acc;         // fixed-point sums, FIXED_WORDS per pixel of every job
    unsigned long long* dropped;
    unsigned long long* claim;       // next padded path index
    uint32_t capacity;               // path slots
    uint32_t* pw;                    // state records, [slot][128]: path words, then lane words
    uint32_t* queues;                // [queue][capacity]
    uint32_t* counts;                // [queue]
    int blocks;
};
cudaError_t launch_wavefront_start_exact(const WaveLaunch& l, cudaStream_t stream);
cudaError_t launch_wavefront_start_fast(const WaveLaunch& l, cudaStream_t stream);
cudaError_t launch_wavefront_iteration_exact(const WaveLaunch& l, int parity, cudaStream_t stream);
cudaError_t launch_wavefront_iteration_fast(const WaveLaunch& l, int parity, cudaStream_t stream);
int wavefront_blocks_per_sm_exact();
int wavefront_blocks_per_sm_fast();

// Rounds fixed-point sums to f64 (out = sum, or out += sum with `accumulate`), one
// thread per pixel component.
cudaError_t launch_fixed_to_f64(const unsigned long long* acc, double* out, uint64_t n_pixels, int accumulate,
                                cudaStream_t stream);
// Brilliance, fire and scintillation of every view (`sums`: the batch's f64 per-pixel
// sums; jobs 2v and 2v + 1 are view v's two half-sample renders, at their out_offset)
// into out[3 * v] (ix_design.h).
cudaError_t launch_image_metrics(const ix_scene* scenes, const BatchJob* jobs, uint32_t n_views, const double* sums,
                                 float* out, cudaStream_t stream);

// Per-function check kernels: evaluate one reference function per input row on the
// device so the host can compare against the CPU oracle value by value.
enum CheckFn {
    CHECK_SAMPLE_DRAWS = 0,   // in: pixel, sample (u32)  out: seed (u32 bits), jx, jy, hero
    CHECK_HERO_LAMBDAS = 1,   // in: hero_rand           out: 8 wavelengths
    CHECK_DISPERSION = 2,     // in: lambda               out: n (scene material)
    CHECK_CMF = 3,            // in: lambda               out: x, y, z
    CHECK_D65 = 4,            // in: lambda               out: power
    CHECK_EXP_LANE = 5,       // in: x                    out: exp
    CHECK_TIR_DELTA = 6,      // in: n1, cos_i, sin_i     out: delta
    CHECK_FRESNEL = 7,        // in: n1, n2, cos_i, I,Q,U,V  out: reflected I,Q,U,V, rs, rp
    CHECK_ENV = 8,            // in: dir xyz, lambda, observer xyz  out: radiance
    CHECK_INTERSECT = 9,      // in: origin xyz, dir xyz  out: t, facet (as float)
    CHECK_TRACE = 10,         // in: pixel, sample (u32)  out: x, y, z, bounces
    CHECK_CAMERA_RAY = 11,    // in: pixel, sample (u32)  out: origin xyz, dir xyz
    CHECK_ABSORPTION = 12,    // in: lambda               out: alpha (abs_o)
    CHECK_TRACE_RAY = 13,     // in: origin xyz, dir xyz, seed (u32), hero  out: x, y, z, bounces
    CHECK_STOKES_ROTATE = 14, // in: k xyz, n xyz, prev_pn xyz, has_prev (u32), I,Q,U,V
                              // out: rotated I,Q,U,V, the new plane normal xyz
    CHECK_FRESNEL_CHANNEL = 15,  // in: n1, n2, cos_i, I,Q,U,V  out: reflected I,Q,U,V,
                                 // transmitted I,Q,U,V, r_s, r_p, t_s, t_p, TIR (0 / 1)
    CHECK_CHANNEL_ALPHA = 16, // in: k xyz, lambda  out: alpha (scene material, isotropic form)
    CHECK_BIAXIAL = 17,       // in: k xyz, normal xyz, cos_i, lambda, n_beta  out: the scene
                              // material's biaxial indicatrix at n_beta (its absorption at
                              // lambda): wave_indices (slow, fast), eigen D
                              // (slow xyz, fast xyz), mode_poynting_dir (slow, fast),
                              // resolve_entry_mode (slow n, dir xyz, fast n, dir xyz), assigned-
                              // mode alpha of the trichroic tensor (mode B, mode A)
};

struct CheckLaunch {
    ix_scene scene;    // device planes
    uint32_t flags;    // scene_flags(scene)
    int fn;
    uint32_t n;
    uint32_t in_stride;   // 32-bit words per input row
    uint32_t out_stride;  // 32-bit words per output row
    const uint32_t* in;   // device
    uint32_t* out;        // device
};

// Analytic optical metrics (ix_metrics.cu): one CTA per pose.
struct MetricsStoneDev {
    uint32_t plane_offset;  // first float4 of the stone in `planes`
    uint32_t n_planes;
    float half_width;       // girdle half-width (fan.rs:34), measured on the host in f64
    ix_dispersion dispersion;
};
struct MetricsPoseDev {
    uint32_t stone;
    float basis[6][9];  // forward, right, up of the pose and of its 5 yaw-jittered poses
};
struct MetricsLaunch {
    const float4* planes;          // device
    const MetricsStoneDev* stones;  // device
    const MetricsPoseDev* poses;    // device
    uint32_t n_poses;
    uint32_t want_fire;             // fire and scintillation rays traced
    ix_environment env;             // the scoring light: exposure 1, no tray, default shadow
    float spec;                     // its spectral power at 550 nm
    float factor;                   // threshold over the median hemisphere radiance
    float head_shadow_cos;          // observer cone (visibility.rs:16)
    float dirs[96][3];              // hemisphere probe directions (lighting.rs:74)
    float* out;                     // device, 5 floats per pose
};
cudaError_t launch_metrics_exact(const MetricsLaunch& l, cudaStream_t stream);
cudaError_t launch_metrics_fast(const MetricsLaunch& l, cudaStream_t stream);

// Spectral attribution of a trace launch (classify_path, color/metrics/attribution.rs:75):
// the exit lighting that decides the classes, and where each sample's class code and
// luminance go -- [sample][pixel] over the launch's samples [0, spp) and pixels
// [0, n_pixels), so the fold reads them coalesced.
struct AttrLaunch {
    ix_environment env;     // the scoring light: exposure 1, no tray, default shadow
    float spec;             // its spectral power at 550 nm
    float factor;           // threshold over the median hemisphere radiance
    float head_shadow_cos;  // observer cone (visibility.rs:16)
    float dirs[96][3];      // hemisphere probe directions (lighting.rs:74)
    uint8_t* cls;           // device, spp * n_pixels class codes (IX_CLASS_*, IX_CLASS_MISS)
    float* y;               // device, spp * n_pixels luminances (the sample's XYZ.y)
};
// AttributionPixel::add (renderer/attribution_map.rs:105) of a launch's records, in
// ascending sample order, into `map` (device, n_pixels records of the launch's pixels).
struct AttrFoldLaunch {
    const uint8_t* cls;
    const float* y;
    ix_attribution_pixel* map;
    uint32_t n_pixels;
    uint32_t spp;
};
cudaError_t launch_trace_attributed_exact(const TraceLaunch& l, const AttrLaunch& a, cudaStream_t stream);
cudaError_t launch_trace_attributed_fast(const TraceLaunch& l, const AttrLaunch& a, cudaStream_t stream);
int trace_attributed_blocks_per_sm_exact(int threads, int uniaxial);
int trace_attributed_blocks_per_sm_fast(int threads, int uniaxial);
cudaError_t launch_attribution_fold_exact(const AttrFoldLaunch& l, cudaStream_t stream);
cudaError_t launch_attribution_fold_fast(const AttrFoldLaunch& l, cudaStream_t stream);

cudaError_t launch_trace_exact(const TraceLaunch& l, cudaStream_t stream);
cudaError_t launch_trace_fast(const TraceLaunch& l, cudaStream_t stream);
cudaError_t launch_batch_exact(const BatchLaunch& l, cudaStream_t stream);
cudaError_t launch_batch_fast(const BatchLaunch& l, cudaStream_t stream);
int batch_blocks_per_sm_exact(int threads, int variant, int uniaxial);
int batch_blocks_per_sm_fast(int threads, int variant, int uniaxial);
// The path-pool kernels (ix_pool.cu), dispatched to by launch_trace_* / launch_batch_*
// for the pool shapes.  A variant a build does not carry returns cudaErrorInvalidValue
// (the exact build carries the 128-thread pool shape only).
cudaError_t launch_pool_trace_exact(const TraceLaunch& l, cudaStream_t stream);
cudaError_t launch_pool_trace_fast(const TraceLaunch& l, cudaStream_t stream);
cudaError_t launch_pool_batch_exact(const BatchLaunch& l, cudaStream_t stream);
cudaError_t launch_pool_batch_fast(const BatchLaunch& l, cudaStream_t stream);
int pool_trace_blocks_per_sm_exact(int variant, int uniaxial);
int pool_trace_blocks_per_sm_fast(int variant, int uniaxial);
int pool_batch_blocks_per_sm_exact(int variant, int uniaxial);
int pool_batch_blocks_per_sm_fast(int variant, int uniaxial);
cudaError_t launch_check_exact(const CheckLaunch& l, cudaStream_t stream);
cudaError_t launch_check_fast(const CheckLaunch& l, cudaStream_t stream);
// Occupancy-derived resident blocks per SM for the trace kernel at `threads` per block.
// In these `uniaxial` is the transport class (TransportClass) of the instantiation.
int trace_blocks_per_sm_exact(int threads, int variant, int uniaxial, size_t* smem_bytes);
int trace_blocks_per_sm_fast(int threads, int variant, int uniaxial, size_t* smem_bytes);
// FP32 FMA-pipe throughput probe (ix_probe.cu): best FLOP/s of `reps` timed runs.
cudaError_t fp32_probe(int sm_count, int reps, cudaStream_t stream, double* flops);

// ix_scene_routes_to_gpu for a scene whose arrays live in device memory (the device
// entries): the tools are counted but not read on the host -- the caller validates them
// with ix_tool_validate before uploading them.
inline int routes_device_scene(const ix_scene* s) {
    if (!s) return 0;
    if (s->n_tools > IX_MAX_TOOLS || (s->n_tools && !s->tools)) return 0;
    ix_scene copy = *s;
    copy.tools = nullptr;
    copy.n_tools = 0;
    return ix_scene_routes_to_gpu(&copy);
}

}  // namespace ix
