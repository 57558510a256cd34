/*
 * ix_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * The C entry points of the CPU oracle: a restatement, in C++, of the reference's CPU
 * spectral tracer (crates/indicatrix/src/optics/raytracer, renderer/cpu_frame.rs).
 * Only the test suite, the smoke check and the benchmark's CPU-baseline leg load this
 * library, and only as the checker / reported baseline; the CUDA backend never links it.
 */
#ifndef IX_ORACLE_H
#define IX_ORACLE_H

#include <stdint.h>
#include "../include/ix_scene.h"
#include "../include/ix_attribution.h"
#include "../include/ix_display.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-path bookkeeping a test can read beside the XYZ result. */
typedef struct ixo_path_info {
    uint32_t bounces;       /* loop iterations run                                   */
    uint32_t termination;   /* 0 escaped, 1 russian roulette, 2 hit the bounce cap     */
    uint32_t escaped;       /* the path's own environment lookup ran                   */
    uint32_t exit_splits;   /* exit-split probes that reached the environment          */
} ixo_path_info;

/* What one traced path did (PathEvents, transport/path_events.rs:27-49): filled by the
 * same hook points the reference's recorder uses (bounce_body.rs:388, :680 and
 * attributed.rs:61).  first_facet / exit_facet are -1 when absent. */
typedef struct ixo_path_events {
    int32_t first_facet;
    uint32_t first_entered;      /* the first facet event left the ray inside the stone */
    int32_t exit_facet;          /* the first inside-to-outside transition              */
    float exit_normal[3];        /* its facet's outward normal                           */
    float exit_dir[3];           /* the ray direction after it                           */
    uint32_t exit_bounce;
    uint32_t bounces_before_exit;
    uint32_t reentered;
    uint32_t termination;        /* ixo_path_info numbering                              */
    uint32_t has_escaped_dir;
    float escaped_dir[3];
    uint32_t scattered;          /* a Henyey-Greenstein scattering event happened         */
} ixo_path_events;
typedef struct ixo_flop_counts {
    uint64_t add, mul, fma, div, sqrt, transcendental, paths;
} ixo_flop_counts;

/* sampling.rs */
uint32_t ixo_hash_u32(uint32_t x);
float ixo_low_discrepancy_base2(uint32_t n);
float ixo_radical_inverse_base(uint32_t n, uint32_t base);
void ixo_pixel_rotations(uint32_t pixel, float out[3]);
void ixo_sample_draws(uint32_t pixel, uint32_t sample, const float rot[3], uint32_t* seed,
                      float out[3]);
/* camera.rs */
void ixo_camera_new(float yaw, float pitch, float distance, float fov_deg, ix_camera* out);
void ixo_generate_ray(const ix_camera* cam, float sx, float sy, float w, float h, float jx,
                      float jy, float origin[3], float dir[3]);
/* transport/mod.rs:58 */
void ixo_hero_wavelengths(float hero_rand, float out[8]);
/* dispersion.rs:170 */
float ixo_dispersion_eval(const ix_dispersion* d, float lambda_nm);
/* color/cie1931.rs:157, environment/spectral.rs:28 */
void ixo_cmf(float lambda_nm, float out[3]);
float ixo_d65(float lambda_nm);
/* simd/exp_poly.rs:37 */
float ixo_exp_lane(float x);
/* polarization.rs + refraction/tir.rs: Fresnel amplitude coefficients and TIR phase */
float ixo_tir_phase_delta(float n1, float cos_i, float sin_i);
void ixo_fresnel_reflect_apply(float r_s, float r_p, const float s_in[4], float s_out[4]);
/* spectral_absorption: alpha(lambda) of one eigenmode (Gaussian bands + the spline). */
float ixo_spectral_absorption(const ix_absorption* a, float lambda_nm);
/* rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:69) as facet_event calls
 * it: the new plane-of-incidence normal normalize_or_zero(k x n) and, when there is a
 * previous one, the Stokes vector rotated by frame_rotation(psi). */
void ixo_rotate_stokes(const float k[3], const float normal[3], const float prev_pn[3], uint32_t has_prev,
                       const float s_in[4], float s_out[4], float cpn_out[3]);
/* One channel's Fresnel step at (n1, n2, cos_i): out[0..3] the reflected Stokes vector
 * (the TIR retarder past the critical angle), out[4..7] the transmitted one, out[8..11]
 * r_s, r_p, t_s, t_p, out[12] 1 for TIR (then out[4..11] are 0). */
void ixo_fresnel_channel(float n1, float n2, float cos_i, const float s_in[4], float out[13]);
/* A non-birefringent material's channel alpha along wave normal k
 * (channel_absorption_alphas_assigned, raytracer/absorption.rs:197). */
float ixo_channel_alpha(const ix_material* m, const float k[3], float lambda_nm);
int ixo_tool_ray_interval(const ix_tool* t, const float origin[3], const float dir[3], float out[2]);
int ixo_tool_contains(const ix_tool* t, const float p[3]);
float ixo_tool_boundary_gap(const ix_tool* t, const float p[3]);
void ixo_tool_outward_normal(const ix_tool* t, const float p[3], float out[3]);
int ixo_intersect_stone(const float* planes, uint32_t n_planes, const ix_tool* tools, uint32_t n_tools,
                        const float origin[3], const float dir[3], float* t, float normal[3], int32_t* facet,
                        int32_t* entering);
void ixo_biaxial_bundle(const ix_material* m, const float k[3], const float normal[3], float cos_i,
                        float lambda_nm, float n_beta, float out[24]);
/* DaylightSun next-event estimation (environment/nee.rs:81,144; scattering/mod.rs:102;
 * scattering/frosted.rs:98). */
float ixo_sun_nee_sample(const ix_environment* env, float u0, float u1, float dir[3]);
float ixo_sun_nee_pdf(const ix_environment* env, const float dir[3]);
float ixo_balance_heuristic(float a, float b);
void ixo_frosted_sun_nee(const ix_scene* sc, const float origin[3], const float ext_normal[3], uint32_t seed,
                         uint32_t bounce, const float lambdas[8], const float intensities[8], float radiance[8]);
/* simd/slab.rs:147 + intersect.rs:101: returns 1 and fills t/idx on a hit */
int ixo_intersect(const float* planes, uint32_t n_planes, const float origin[3],
                  const float dir[3], float* t, int32_t* facet);
/* Environment construction (environment/mod.rs, optics/studio_rig.rs, color.rs) for the
 * reference's LightingPreset index (environment/mod.rs:475-493).  Returns 0 on success,
 * -1 for a preset this oracle does not model. */
int ixo_environment_preset(int32_t preset_index, float exposure, float light_yaw,
                           float light_pitch, float backdrop, float surface_glare,
                           float head_shadow_deg, ix_environment* out);
void ixo_environment_uniform(float radiance, ix_environment* out);
/* Escape radiance of one channel (environment/rig.rs:18-49). */
float ixo_environment_channel(const ix_environment* env, const float dir[3], float lambda_nm,
                              const float observer[3]);
/* trace_spectral_ray (transport/mod.rs:118): one path from an explicit ray. */
int ixo_trace_ray(const ix_scene* scene, const float origin[3], const float dir[3],
                  uint32_t seed, float hero_rand, float xyz[3], ixo_path_info* info);
/* One (pixel, absolute sample) exactly as renderer/cpu_frame.rs:45 traces it. */
int ixo_trace_sample(const ix_scene* scene, uint32_t pixel, uint32_t sample, float xyz[3],
                     ixo_path_info* info);
/* trace_pixels_interleaved (renderer/cpu_frame.rs:104) for every pixel of the frame,
 * partitioned over `threads` host threads by the same interleaved stride.  Writes the
 * reference's f32 per-pixel sums (ascending sample order, non-finite samples dropped)
 * into sums_f32 and the same samples summed in f64 into sums_f64 (either may be NULL).
 * Returns the number of dropped non-finite samples, or -1 on an unsupported scene. */
int64_t ixo_trace_frame(const ix_scene* scene, uint32_t sample_offset, uint32_t spp,
                        uint32_t threads, float* sums_f32, double* sums_f64);
/* Like ixo_trace_frame but only for the pixels [pixel_begin, pixel_end). */
int64_t ixo_trace_pixels(const ix_scene* scene, uint32_t pixel_begin, uint32_t pixel_end,
                         uint32_t sample_offset, uint32_t spp, uint32_t threads,
                         double* sums_f64);
/* A set of (scene, pixel) entries, each traced over samples [sample_offset,
 * sample_offset + spp[k]) as renderer/cpu_frame.rs:45 traces them, entries claimed one at
 * a time by `threads` host threads.  Per-entry f64 sums go to sums_f64 (3 per entry) when
 * it is not NULL.  Returns the dropped non-finite samples, or -1 on an unsupported scene
 * or an out-of-range entry. */
int64_t ixo_trace_pixel_set(const ix_scene* scenes, uint32_t n_scenes, const uint32_t* scene_of,
                            const uint32_t* pixel, const uint32_t* spp, uint32_t n, uint32_t sample_offset,
                            uint32_t threads, double* sums_f64);
/* 1 for the build with the AVX2 twins of the slab scan and the 8-lane exp (simd/slab.rs,
 * simd/exp_poly.rs), 0 for the scalar build. */
int ixo_simd_build(void);
/* Per-sample XYZ of the pixels [pixel_begin, pixel_end) x samples, row-major
 * [pixel][sample][3], for path-level comparisons. */
int ixo_trace_samples(const ix_scene* scene, uint32_t pixel_begin, uint32_t pixel_end,
                      uint32_t sample_offset, uint32_t spp, uint32_t threads, float* xyz,
                      uint32_t* bounces);
/* StandardGemCuts::standard_round_brilliant (geometry/cuts/round_brilliant.rs:71-155),
 * the reference's fixed test stone, restated in f32 exactly as built there.
 * Writes 74 x {nx, ny, nz, d} (57 facets plus 16 girdle planes and the culet). */
uint32_t ixo_standard_round_brilliant(float* out);
/* evaluate_gem_optical_metrics (color/metrics/evaluate.rs:158) for a camera pose and a
 * lighting preset (LightingPreset index, light yaw/pitch, head-shadow degrees).  Writes
 * {brilliance_pct, fire_index, scintillation_pct, windowing_pct, extinction_pct}.
 * Returns 0, or -1 for an unmodelled preset or an empty plane set. */
int ixo_metrics(const float* planes, uint32_t n_planes, const ix_material* material, float cam_yaw,
                float cam_pitch, int32_t preset, float light_yaw, float light_pitch,
                float head_shadow_deg, float out[5]);
/* Pieces of the metrics setup, for unit checks: the fan's girdle half-width
 * (fan.rs:34, measure_model_width in f64) and the exit lighting's threshold and
 * head-shadow cone cosine (lighting.rs:137, visibility.rs:16). */
float ixo_metrics_half_width(const float* planes, uint32_t n_planes);
int ixo_metrics_lighting(int32_t preset, float light_yaw, float light_pitch, float head_shadow_deg,
                         float out[3]);
/* trace_spectral_ray_attributed_soa_geom (transport/attributed.rs:28): ixo_trace_ray plus
 * the path's events. */
int ixo_trace_ray_events(const ix_scene* scene, const float origin[3], const float dir[3],
                         uint32_t seed, float hero_rand, float xyz[3], ixo_path_events* events);
/* The recorder alone, for its unit checks: PathEvents::default and PathEvents::facet
 * (path_events.rs:55) for a facet event of `facet` with outward `normal`. */
void ixo_path_events_reset(ixo_path_events* events);
void ixo_path_events_facet(ixo_path_events* events, uint32_t bounce, int32_t facet, const float normal[3],
                           uint32_t inside_before, uint32_t inside_after, const float dir_after[3]);
/* classify_path (color/metrics/attribution.rs:75) through class_index
 * (renderer/attribution_map.rs:39) under the exit lighting of a LightingPreset index,
 * light yaw / pitch and head-shadow degrees (lighting.rs:137): the class slot
 * (IX_CLASS_*), IX_CLASS_MISS for a path with no facet event, or -1 for an unmodelled
 * preset.  `observer` is the unit direction from the stone to the eye. */
int ixo_classify_path(const ixo_path_events* events, const float observer[3], int32_t preset,
                      float light_yaw, float light_pitch, float head_shadow_deg);
/* AttributionPixel::add (attribution_map.rs:105) for one sample (class IX_CLASS_MISS for a
 * miss; scattered / fluoresced flags). */
void ixo_attribution_add(ix_attribution_pixel* pixel, uint32_t class_code, uint32_t scattered,
                         uint32_t fluoresced, float y);
/* The attributed frame loop: for the pixels [pixel_begin, pixel_end) and samples
 * [sample_offset, sample_offset + spp), each sample traced as renderer/cpu_frame.rs:45
 * traces it with its events recorded, classified under the given lighting and added to
 * map[pixel - pixel_begin] in ascending sample order.  Per-pixel XYZ sums (f64, finite
 * samples) are added into sums_f64 when it is not NULL.  Returns the number of dropped
 * non-finite samples, or -1 on an unsupported scene or an unmodelled preset. */
int64_t ixo_attribute_pixels(const ix_scene* scene, int32_t preset, float light_yaw,
                             float light_pitch, float head_shadow_deg, uint32_t pixel_begin,
                             uint32_t pixel_end, uint32_t sample_offset, uint32_t spp,
                             uint32_t threads, ix_attribution_pixel* map, double* sums_f64);
/* 1 when this build counts floating-point operations. */
int ixo_counting_build(void);
/* Counting build only: trace the given pixels x samples and return the operation tally. */
int ixo_count_flops(const ix_scene* scene, uint32_t pixel_begin, uint32_t pixel_end,
                    uint32_t pixel_step, uint32_t sample_offset, uint32_t spp,
                    ixo_flop_counts* out);

/* The display pipeline after the path (renderer/guide_pass.rs, renderer/denoise/,
 * renderer/tonemap.rs, renderer/frame_denoise.rs); threads 0 = all host threads, the
 * results do not depend on it. */
/* shading_normal_near_edge (optics/raytracer/intersect.rs:196). */
void ixo_shading_normal_near_edge(const float* planes, uint32_t n_planes, const float hit_point[3], int32_t facet,
                                  const float hit_normal[3], float radius, float out[3]);
void ixo_atrous_params_default(ix_atrous_params* p);
/* Counting build only: the operation tally of one A-Trous denoise (paths = pixel-passes). */
int ixo_count_denoise_flops(const float* color, const float* depth, const float* normal, const int32_t* facet_id,
                            const uint32_t* path_sig, uint32_t width, uint32_t height, uint32_t spp,
                            const ix_atrous_params* params, ixo_flop_counts* out);
void ixo_generate_guide_buffers(uint32_t width, uint32_t height, const ix_camera* cam, const float* planes,
                                uint32_t n_planes, float n_d, float* depth, float* normal, int32_t* facet_id,
                                uint32_t* path_sig, int threads);
float ixo_n_d(const ix_dispersion* d);
void ixo_atrous_denoise(const float* color, const float* depth, const float* normal, const int32_t* facet_id,
                        const uint32_t* path_sig, uint32_t width, uint32_t height, uint32_t spp,
                        const ix_atrous_params* params, float* out, int threads);
void ixo_color_encode(const float xyz[3], uint32_t color_space, uint8_t out[4]);
void ixo_tonemap_to_rgba(const float* xyz, uint64_t pixels, float scale, uint32_t color_space, uint8_t* rgba,
                         int threads);
void ixo_denoise_and_tonemap_frame(uint32_t width, uint32_t height, uint32_t spp, const float* accum,
                                   const float* depth, const float* normal, const int32_t* facet_id,
                                   const uint32_t* path_sig, const ix_atrous_params* params, uint8_t* rgba,
                                   int threads);

#ifdef __cplusplus
}
#endif
#endif
