/*
 * ix_cuda.h -- C ABI of libix_cuda.so, the B200 (sm_100a) backend for indicatrix's
 * Path-Traced spectral sample loop.
 *
 * The entry points are what a host binding of the reference's `GpuBackend`
 * (crates/indicatrix/src/renderer/gpu_backend/backend.rs, stub.rs) would call: plain
 * pointers and sizes, no CUDA or torch types except an opaque stream handle on the
 * device-resident entry.  Each declaration cites the reference interface it replaces.
 *
 * Contract shared by every accumulate entry (gpu_backend/mod.rs:24-31, :122-164):
 *   - `accum_xyz` is caller-owned, row-major, width * height * 3; the backend ADDS the
 *     per-pixel sums of samples [sample_offset, sample_offset + spp) into it, and only
 *     when it returns IX_DONE;
 *   - IX_DECLINED leaves `accum_xyz` untouched and means "trace the full spp on the
 *     CPU"; device errors are reported as a decline and mark the backend lost;
 *   - IX_CANCELLED leaves `accum_xyz` untouched; `cancel` (may be NULL) is the caller's
 *     one-byte flag -- a Rust AtomicBool through AtomicBool::as_ptr -- read as nonzero =
 *     cancelled, polled between launches;
 *   - a sample whose XYZ has a NaN/Inf component is dropped but still counted
 *     (optics/raytracer/sampling.rs:237).
 * Per-pixel sums are formed on the device in f64 and are bit-identical for any chunking
 * and any run.  (The path-pool kernels form them exactly, in fixed point, and round
 * once; a sample with a component of 2^62 or more is dropped and counted as a non-finite
 * one is.)
 */
#ifndef IX_CUDA_H
#define IX_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "ix_attribution.h"
#include "ix_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

/* GpuAccumulate (gpu_backend/mod.rs:308-326). */
enum { IX_DONE = 0, IX_DECLINED = 1, IX_CANCELLED = 2 };
/* GpuPipelineKind (gpu_backend/mod.rs:347-353). */
enum { IX_PIPELINE_MEGAKERNEL = 0, IX_PIPELINE_WAVEFRONT = 1 };
/* Rounding of the transport kernels: FAST lets the compiler fuse multiply-adds;
 * EXACT rounds every step as the reference's CPU code does (no contraction). */
enum { IX_PRECISION_FAST = 0, IX_PRECISION_EXACT = 1 };

typedef struct ix_backend ix_backend;

typedef struct ix_backend_options {
    int32_t device;              /* CUDA device ordinal                                  */
    uint32_t pipeline;           /* IX_PIPELINE_*                                        */
    uint32_t precision;          /* IX_PRECISION_*                                       */
    uint32_t threads_per_block;  /* CTA size of batch plans: 0 = any (autotuned), or 64,  */
                                 /* 128 or 256 (the path-pool loop at that size); any     */
                                 /* other value makes ix_backend_create return NULL       */
    uint64_t chunk_paths;        /* paths per launch; 0 = default (2^26)                   */
    uint32_t kernel_variant;     /* kernel of single-scene calls: 0 default (the path-pool */
                                 /* loop, 128 threads, 32 warps/SM budget); k = 1..6 picks  */
                                 /* variant k - 1 (budget + 3 * shape, shapes 0-1 of      */
                                 /* ix_batch_plan_autotune); anything else returns NULL    */
} ix_backend_options;

/* GpuWorkLimits (gpu_backend/limits.rs:6-27): a request above a limit is declined. */
typedef struct ix_work_limits {
    uint64_t max_pixels;
    uint64_t max_paths_per_call;
    uint32_t max_spp;
} ix_work_limits;

/* One stone of a batched request (GpuBatchItem, gpu_backend/mod.rs:246). */
typedef struct ix_batch_item {
    const ix_scene* scene;
    uint32_t sample_offset;
    uint32_t spp;
    double* accum_xyz;           /* width * height * 3, added into on IX_DONE           */
    int32_t status;              /* written by ix_accumulate_batch                      */
} ix_batch_item;

/* Device timing of the last accumulate call on this backend. */
typedef struct ix_timing {
    float kernel_ms;             /* trace kernel(s), CUDA events on the backend stream   */
    float reduce_ms;             /* host-visible copy and fold                           */
    uint64_t paths;
    uint32_t launches;           /* kernels this library launched for the call           */
} ix_timing;

/* GpuBackend::acquire / acquire_with_diagnostics (gpu_backend/limits.rs:50-71).
 * `opts` may be NULL (device 0, megakernel, fast rounding).  Returns NULL when no
 * usable device is present. */
ix_backend* ix_backend_create(const ix_backend_options* opts);
/* Drop of GpuBackend. */
void ix_backend_destroy(ix_backend* b);
/* GpuBackend::adapter_label (backend.rs:165): device name, NUL-terminated. */
int ix_backend_label(const ix_backend* b, char* buf, size_t len);
/* GpuBackend::set_pipeline_kind (backend.rs:165).  IX_PIPELINE_WAVEFRONT makes batch plans
 * created afterwards start on the wavefront pipeline (variant 12 of ix_batch_plan_*: path
 * state in device memory between kernels, one kernel per event queue) when every scene is
 * isotropic; single-scene calls and uniaxial plans run the megakernel either way. */
void ix_set_pipeline_kind(ix_backend* b, uint32_t kind);
/* GpuBackend::set_work_limits (gpu_backend/limits.rs:75). */
void ix_set_work_limits(ix_backend* b, const ix_work_limits* limits);
/* Rounding mode of later calls (IX_PRECISION_*). */
void ix_set_precision(ix_backend* b, uint32_t precision);
/* scene_routes_to_gpu (gpu_backend/mod.rs:288): 1 when this backend can trace `scene`
 * (<= IX_MAX_PLANES planes carved by <= IX_MAX_TOOLS valid tools, polished or frosted
 * facets, an isotropic, uniaxial or biaxial material with modelled dispersion, a lighting
 * model of the reference's six (not a UV lamp's line spectrum), at most 2^32 - 1
 * pixels). */
int ix_scene_routes_to_gpu(const ix_scene* scene);
/* scene_routes_to_gpu_with_tools (gpu_backend/tool_routing.rs:81): ix_scene_routes_to_gpu
 * of the stone carved by `tools` (when ntools > 0; else the scene's own tools): at most
 * IX_MAX_TOOLS, each passing ix_tool_validate. */
int ix_scene_routes_to_gpu_with_tools(const ix_scene* scene, const ix_tool* tools, uint32_t ntools);
/* ToolPrimitive::validate (geometry/tool.rs:360): IX_TOOL_OK, or the first failed check
 * (ToolPrimitiveError, tool.rs:133). */
enum {
    IX_TOOL_OK = 0,
    IX_TOOL_NON_FINITE = 1,
    IX_TOOL_NON_POSITIVE_RADIUS = 2,
    IX_TOOL_AXIS_NOT_UNIT = 3,
    IX_TOOL_UNKNOWN_KIND = 4,
    IX_TOOL_UNKNOWN_SWEEP = 5,
    IX_TOOL_PADDING_NOT_ZERO = 6
};
int ix_tool_validate(const ix_tool* tool);
/* GpuBackend::try_accumulate_geom_cancellable (backend.rs:272) with an f32 accumulator:
 * adds (float)(f64 pixel sum) into accum_xyz.  `tools` / `ntools` are the stone's concave
 * tools (`tools: &[ToolPrimitive]`, tool k facet id n_planes + k); with ntools = 0 the
 * scene's own `tools` apply.  `cancel` may be NULL; it is polled between chunks. */
int ix_accumulate(ix_backend* b, const ix_scene* scene, const ix_tool* tools, uint32_t ntools,
                  uint32_t sample_offset, uint32_t spp, float* accum_xyz, const volatile uint8_t* cancel);
/* The same with an f64 accumulator (no rounding of the pixel sums). */
int ix_accumulate_f64(ix_backend* b, const ix_scene* scene, const ix_tool* tools, uint32_t ntools,
                      uint32_t sample_offset, uint32_t spp, double* accum_xyz, const volatile uint8_t* cancel);
/* GpuBackend::try_accumulate_batch_cancellable (backend.rs:451): every routable item
 * traced in one persistent launch; each item's outcome is written to item->status and,
 * when `on_done` is not NULL, reported as on_done(user, index, status) -- the reference's
 * `on_done: &mut dyn FnMut(usize, GpuAccumulate)` -- once per item, in index order,
 * after that item's accumulator is final (items that are not traced first, before any
 * tracing).  Returns IX_DONE when all items are done. */
typedef void (*ix_batch_done_fn)(void* user, uint32_t index, int32_t status);
int ix_accumulate_batch(ix_backend* b, ix_batch_item* items, uint32_t n_items, const volatile uint8_t* cancel,
                        ix_batch_done_fn on_done, void* user);
/* Batched plans (the reference's batch path, backend.rs:451, as ONE persistent launch
 * over many stones and tilts, replayed from a CUDA graph).  A job is a whole frame of
 * scene `scene` over samples [sample_offset, sample_offset + spp).  Scenes, planes and
 * the job table are uploaded once by ix_batch_plan_create; each ix_batch_plan_run
 * overwrites the plan's device sums (job-major, each job width * height * 3 f64, job j
 * starting at ix_batch_plan_job_offset(j)).  Returns NULL when a scene does not route
 * to the GPU or the device fails. */
typedef struct ix_batch_job {
    uint32_t scene;
    uint32_t sample_offset;
    uint32_t spp;
} ix_batch_job;
typedef struct ix_batch_plan ix_batch_plan;
ix_batch_plan* ix_batch_plan_create(ix_backend* b, const ix_scene* scenes, uint32_t n_scenes,
                                    const ix_batch_job* jobs, uint32_t n_jobs);
/* One persistent launch of every job on `stream` (NULL: the backend's stream); not
 * synchronised.  IX_DONE or IX_DECLINED. */
int ix_batch_plan_run(ix_batch_plan* p, void* stream);
/* The autotuner (the reference picks GpuPipelineKind by hand, gpu_backend/mod.rs:347):
 * times every kernel variant this build carries -- the static task loop and the
 * path-pool loop at 64, 128 and 256 threads per CTA, each under three register budgets
 * (variant = budget + 3 * shape) -- `reps` times on a strided sample of about 1/16 of
 * the plan's work (every job represented), then runs the two fastest, the fastest of each
 * loop (static tasks, path pool) and, for an isotropic plan, the wavefront pipeline
 * (variant 12) on the whole plan once each, keeps the fastest of those and writes it to
 * `chosen`.
 * With ix_backend_options.threads_per_block set, only that CTA size is tried.
 * Returns 0, or -1 on a device error. */
int ix_batch_plan_autotune(ix_batch_plan* p, int reps, uint32_t* chosen);
/* Pins the plan's kernel variant (budget + 3 * shape, or 12 for the wavefront pipeline;
 * see ix_batch_plan_autotune).  Returns 0, or -1 when this build or this plan cannot run
 * it. */
int ix_batch_plan_set_variant(ix_batch_plan* p, uint32_t variant);
/* Copies the plan's sums to host memory (ix_batch_plan_output_size doubles). */
int ix_batch_plan_download(ix_batch_plan* p, double* host_out);
uint64_t ix_batch_plan_output_size(const ix_batch_plan* p);
const double* ix_batch_plan_device_output(const ix_batch_plan* p);
uint64_t ix_batch_plan_paths(const ix_batch_plan* p);
uint32_t ix_batch_plan_variant(const ix_batch_plan* p);
uint64_t ix_batch_plan_job_offset(const ix_batch_plan* p, uint32_t job);
void ix_batch_plan_destroy(ix_batch_plan* p);
/* Device-resident form for callers that keep the scene and the sums in GPU memory:
 * `scene->planes`, `scene->facet_finishes` and `scene->tools` (if any) and `d_accum_xyz` are device
 * pointers (IX_DECLINED for one that is not device or managed memory; the tools are
 * counted but not read on the host, so the caller validates them with ix_tool_validate);
 * the launch is enqueued on `stream` (a cudaStream_t, or NULL for the backend's own
 * stream) and not synchronised.
 * `accumulate` = 1 adds into d_accum_xyz, 0 overwrites it. */
int ix_accumulate_device(ix_backend* b, const ix_scene* scene, uint32_t sample_offset,
                         uint32_t spp, double* d_accum_xyz, int accumulate, void* stream);
/* Allocation-free form of ix_accumulate_device.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc (a host whose own pool or arena owns all
 * device memory, a sandboxed plug-in, a runtime with a fixed memory budget): they pass
 * a scene whose `planes` (and `facet_finishes` and `tools`, if any) are device pointers and a device
 * output `d_accum_xyz`
 * (width * height * 3 doubles, added into when `accumulate` is 1, overwritten when 0),
 * and the call needs no backend object and makes no cudaMalloc, cudaFree or other
 * allocating call.  The kernel's work counters live in a 264-byte array in device
 * memory that every GPU loading this library holds until the process exits.
 *
 * Limits and rules:
 *   - at most IX_NOALLOC_MAX_LAUNCHES launches of 2^26 paths each, i.e. width * height
 *     rounded up to whole pixels per launch must fit in 2^32 paths; larger requests
 *     return IX_NOALLOC_ERR_TOO_LARGE without touching the device;
 *   - the first call on a device (the current device) looks up the array's device
 *     address and the launch shape; make that first call before any stream capture;
 *   - every call shares the one array and clears it on `stream` before its launches, so
 *     calls whose work overlaps on the GPU (different streams, or other threads) race:
 *     serialise them on one stream;
 *   - the work is enqueued on `stream` (NULL: the legacy default stream) and not
 *     synchronised;
 *   - dropped samples are not reported: a sample with a non-finite component is left
 *     out of the sums as everywhere else, and counted only inside the shared array,
 *     which no call reads back (a caller that needs the count uses
 *     ix_accumulate_device and ix_last_dropped).
 * Returns IX_DONE, IX_DECLINED (the scene does not route to the GPU) or an
 * IX_NOALLOC_ERR_* code. */
#define IX_NOALLOC_MAX_LAUNCHES 64
enum { IX_NOALLOC_ERR_ARGS = -1, IX_NOALLOC_ERR_TOO_LARGE = -2, IX_NOALLOC_ERR_CUDA = -3 };
int ix_accumulate_device_noalloc(const ix_scene* scene, uint32_t sample_offset, uint32_t spp,
                                 double* d_accum_xyz, int accumulate, void* stream);
/* GpuBackend::is_lost / try_recover / last_lost_reason (backend.rs:704). */
int ix_is_lost(const ix_backend* b);
int ix_try_recover(ix_backend* b);
int ix_last_error(const ix_backend* b, char* buf, size_t len);
/* Timing of the last call (device events on the backend's stream). */
int ix_last_timing(const ix_backend* b, ix_timing* out);
/* Non-finite samples dropped by the last call. */
uint64_t ix_last_dropped(const ix_backend* b);
/* Measured FP32 FMA-pipe throughput of the device in FLOP/s (FMA = 2), the roofline
 * denominator of the FP32-bound transport kernels.  No reference counterpart. */
int ix_probe_fp32_peak(ix_backend* b, double* flops);

/* Host-side scene construction, the reference's own host formulas:
 * Camera::new (optics/raytracer/camera.rs:108). */
void ix_camera_new(float yaw, float pitch, float distance, float fov_deg, ix_camera* out);
/* EnvironmentSource::Studio for a LightingPreset index (environment/mod.rs:475-493,
 * params :318-411, studio_rig.rs:33, color.rs:277-340): 1 IsoHemisphere, 7 Daylight,
 * 8 Incandescent, 9 IlluminantA, 10 RingLights, 11 DarkSpotlight.  Returns 0, or -1 for
 * a preset this backend does not model. */
int ix_environment_preset(int32_t preset_index, float exposure, float light_yaw,
                          float light_pitch, float backdrop, float surface_glare,
                          float head_shadow_deg, ix_environment* out);
/* A uniform dome of constant spectral radiance (white-furnace environment). */
void ix_environment_uniform(float radiance, ix_environment* out);

/* ---- Analytic optical metrics (color/metrics/evaluate.rs:158-392) -----------------
 * evaluate_gem_optical_metrics on the device: for each camera pose, an 18 x 18 fan of
 * grid cells inside the stone's outline disc, 5 aperture rays per cell traced through
 * the stone at n_D (with n_F / n_C companions for fire) and 5 yaw-jittered rays for the
 * temporal scintillation term, each classified against the exit lighting.  Output is
 * the reference's GemOpticalMetrics, in its order. */
typedef struct ix_gem_metrics {
    float brilliance_pct;
    float fire_index;
    float scintillation_pct;
    float windowing_pct;
    float extinction_pct;
} ix_gem_metrics;

/* The lighting a call scores against: a LightingPreset index (as ix_environment_preset),
 * the rig's light yaw / pitch and the environment's head-shadow size in degrees
 * (16 = the default).  Every preset scores (the ASET view as the iso-hemisphere,
 * color/metrics/lighting.rs:125); an unknown preset declines. */
typedef struct ix_metrics_lighting {
    int32_t preset;
    float light_yaw;
    float light_pitch;
    float head_shadow_deg;
} ix_metrics_lighting;

/* One stone of a batched call: its half-spaces (host, n x {nx, ny, nz, d}) and its
 * ordinary dispersion (n_D, n_F, n_C are evaluated from it). */
typedef struct ix_metrics_stone {
    const float* planes;
    uint32_t n_planes;
    ix_dispersion dispersion;
} ix_metrics_stone;

/* One camera pose (Camera::new yaw / pitch) of stone `stone`. */
typedef struct ix_metrics_pose {
    uint32_t stone;
    float cam_yaw;
    float cam_pitch;
} ix_metrics_pose;

/* evaluate_gem_optical_metrics(planes, material, cam_yaw, cam_pitch, environment)
 * (color/metrics/evaluate.rs:158): one pose.  Returns IX_DONE, or IX_DECLINED (no
 * device, an empty or oversized plane set, an unmodelled preset; `out` untouched). */
int ix_evaluate_gem_optical_metrics(ix_backend* b, const float* planes, uint32_t n_planes,
                                    const ix_material* material, float cam_yaw, float cam_pitch,
                                    const ix_metrics_lighting* lighting, ix_gem_metrics* out);
/* Many poses of many stones under one lighting in one launch (one CTA per pose), the
 * batched form of the reference's pose runs (color/metrics/pose_batch.rs, profile.rs,
 * sweep.rs).  want_fire_and_scintillation = 0 is MetricsWanted::CONSUMED_ONLY (fire and
 * scintillation report the placeholders 25 and 75, their rays are not traced). */
int ix_evaluate_gem_optical_metrics_batch(ix_backend* b, const ix_metrics_stone* stones, uint32_t n_stones,
                                          const ix_metrics_lighting* lighting, const ix_metrics_pose* poses,
                                          uint32_t n_poses, uint32_t want_fire_and_scintillation,
                                          ix_gem_metrics* out);

/* Tilt-performance sweeps over the batched metrics kernel, fire-less
 * (MetricsWanted::CONSUMED_ONLY), all poses of a call in one launch. */
#define IX_PROFILE_ANGLES 19   /* PROFILE_ANGLES_DEG (color/metrics/types.rs:27): 0, 5, ..., 90 */
#define IX_AXIS_TILTS 181      /* TILT_ANGLES_DEG (profile.rs:146): -90, ..., 90 */
/* evaluate_angular_profile_at_azimuth (color/metrics/profile.rs:37): brilliance,
 * extinction and windowing at the 19 camera elevations of PROFILE_ANGLES_DEG, azimuth
 * cam_yaw (radians).  `out`: 3 x 19 floats, the three curves in that order. */
int ix_evaluate_angular_profile_at_azimuth(ix_backend* b, const float* planes, uint32_t n_planes,
                                           const ix_material* material, float cam_yaw,
                                           const ix_metrics_lighting* lighting, float* out);
/* evaluate_full_axis_profile_at_azimuth (profile.rs:200) for each of n_axes positive
 * azimuths (degrees): `out` is n_axes x 3 x 181 floats, the brilliance, extinction and
 * windowing curves indexed by tilt away from table-up + 90 degrees.  With the azimuths
 * {0, 45, 90, 135} (PROFILE_AZIMUTHS_DEG) this is evaluate_all_axes_profiles
 * (sweep.rs:74): 724 poses. */
int ix_evaluate_axis_profiles(ix_backend* b, const float* planes, uint32_t n_planes, const ix_material* material,
                              const float* azimuths_deg, uint32_t n_axes, const ix_metrics_lighting* lighting,
                              float* out);

/* ix_accumulate_f64 with spectral attribution: every sample is traced as the plain entry
 * traces it (the same XYZ bits) with its hero path's events recorded
 * (trace_spectral_ray_attributed_soa_geom, transport/attributed.rs:28), labelled by
 * classify_path (color/metrics/attribution.rs:75) under the exit lighting `lighting`
 * describes -- the preset, light pose and head shadow the scene's environment was built
 * from -- and added to its pixel's record with AttributionPixel::add
 * (renderer/attribution_map.rs:105), in ascending sample order.  `attribution` is
 * caller-owned, width * height records, updated only when the call returns IX_DONE.  A
 * frame of more than IX_ATTRIBUTION_MAX_PIXELS pixels (or a NULL map) is traced without
 * attribution (AttributionMap::checked, attribution_map.rs:201).  A scattering stone's
 * records also count the hits whose path scattered; a path ended by its scattering
 * event's roulette (ScatterAbsorbed) takes the roulette's class.  IX_DECLINED also for an
 * unknown lighting preset. */
int ix_accumulate_attributed(ix_backend* b, const ix_scene* scene, const ix_metrics_lighting* lighting,
                             uint32_t sample_offset, uint32_t spp, double* accum_xyz,
                             ix_attribution_pixel* attribution, const volatile uint8_t* cancel);

/* Per-function check kernels (the GPU equivalence harness's Tier-1/Tier-2 units,
 * renderer/gpu/ulp.rs): evaluates function `fn` (ix::CheckFn numbering) for `n` input
 * rows of `in_stride` 32-bit words on the device, writing `out_stride` words per row.
 * `scene` supplies the material, environment and planes.  Host buffers. */
int ix_debug_check(ix_backend* b, const ix_scene* scene, int32_t fn, uint32_t n,
                   const uint32_t* in, uint32_t in_stride, uint32_t* out, uint32_t out_stride);

#ifdef __cplusplus
}
#endif

#endif /* IX_CUDA_H */
