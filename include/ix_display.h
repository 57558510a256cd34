/*
 * ix_display.h -- the display pipeline after the path: guide-buffer prepass, edge-avoiding
 * A-Trous denoise and tone-mapping to RGBA8, as C-ABI entry points of libix_cuda.so.
 *
 * Reference interfaces replaced (crates/indicatrix/src/renderer/, paths in the project):
 *   guide_pass.rs:120-160  generate_guide_buffers[_with_index]  -> ix_generate_guide_buffers
 *   denoise/mod.rs:280-330 AtrousDenoiser::denoise_into          -> ix_atrous_denoise
 *   tonemap.rs:98-128      tonemap_to_rgba_with_threads_into     -> ix_tonemap_to_rgba
 *   tonemap.rs:213-231     tonemap_accumulation                  -> ix_tonemap_accumulation
 *   frame_denoise.rs:40-80 denoise_and_tonemap_frame[_with_params]_into
 *                                                                 -> ix_denoise_and_tonemap_frame
 *   (this library's own)   guides + average + denoise + tone-map of one accumulated frame,
 *                          every step on the device, guides cached per camera pose and
 *                          stone                                   -> ix_display_frame
 *
 * Buffers are host pointers, row-major (index = y * width + x); a Vec3 buffer is three
 * floats per pixel (x, y, z), RGBA8 is four bytes per pixel.  Every call returns IX_DONE
 * (0) or IX_DECLINED (1, nothing written; ix_last_error says why) like the transport
 * entries of ix_cuda.h, and takes the backend's FIFO turn.
 */
#ifndef IX_DISPLAY_H
#define IX_DISPLAY_H

#include <stdint.h>

#include "ix_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

/* AtrousParams (denoise/mod.rs:157-203).  ix_atrous_params_default() gives the
 * reference's defaults: 5 passes, sigma_color 0.35, sigma_depth 0.1, normal_power 64,
 * taper_reference_spp 4, taper_identity_epsilon 0.02. */
typedef struct ix_atrous_params {
    uint32_t num_passes;          /* clamped to 1..=8; stride 1 << pass                  */
    float sigma_color;            /* XYZ distance sigma at spp = 0, before the taper      */
    float sigma_depth;
    float normal_power;           /* max(0, dot)^normal_power                            */
    float taper_reference_spp;    /* N0 of taper(spp) = 1 / sqrt(1 + spp / N0)           */
    float taper_identity_epsilon; /* taper below this: exact identity copy               */
} ix_atrous_params;

/* ColorSpace (color/space.rs:126-141). */
enum {
    IX_COLOR_SPACE_SRGB = 0,
    IX_COLOR_SPACE_DISPLAY_P3 = 1,
    IX_COLOR_SPACE_REC2020 = 2,
    IX_COLOR_SPACE_ACESCG = 3
};

/* Device time of the last display call's stages (CUDA events on the stream it ran on):
 * the guide pass (0 when the cache served it), packing, and the A-Trous passes with the
 * fused tone-map; `atrous_passes` of the `launches` kernels were A-Trous passes. */
typedef struct ix_display_timing {
    float guide_ms;
    float pack_ms;
    float atrous_ms;
    uint32_t atrous_passes;
    uint32_t launches;
} ix_display_timing;

struct ix_backend;

void ix_atrous_params_default(ix_atrous_params* out);
int ix_display_last_timing(const struct ix_backend* b, ix_display_timing* out);

/* One un-jittered camera ray per pixel (guide_pass.rs:640-690): first-hit depth t
 * (1e6 on a miss), facet normal (0 on a miss, 3 floats per pixel), facet id (-1 on a
 * miss) and, for n_d > 1, the interior path signature (guide_pass.rs:560-625; 0 on a
 * miss and everywhere when n_d <= 1 or NaN).  `path_sig` may be NULL. */
int ix_generate_guide_buffers(struct ix_backend* b, uint32_t width, uint32_t height,
                              const ix_camera* camera, const float* planes, uint32_t n_planes,
                              float n_d, float* depth, float* normal, int32_t* facet_id,
                              uint32_t* path_sig);

/* AtrousDenoiser::denoise_into: `color` is the averaged XYZ (accumulation / spp), the
 * guides as ix_generate_guide_buffers writes them, `path_sig` NULL for no signature
 * term.  `out` (width * height * 3 floats) may not alias `color`. */
int ix_atrous_denoise(struct ix_backend* b, const float* color, const float* depth,
                      const float* normal, const int32_t* facet_id, const uint32_t* path_sig,
                      uint32_t width, uint32_t height, uint32_t spp,
                      const ix_atrous_params* params, float* out);

/* tonemap_to_rgba_with_threads_into: each XYZ value times `scale` through
 * xyz_to_srgb_gamma (optics/raytracer/color.rs:415) into `pixels` RGBA8 texels. */
int ix_tonemap_to_rgba(struct ix_backend* b, const float* xyz, uint64_t pixels, float scale,
                       uint8_t* rgba);

/* tonemap_accumulation: summed XYZ of `samples_per_pixel` samples to RGBA8 in
 * `color_space` (ColorSpace::encode with AcesFilmic exposure 1, color/space.rs:234). */
int ix_tonemap_accumulation(struct ix_backend* b, uint32_t width, uint32_t height,
                            uint32_t samples_per_pixel, const float* accum, uint32_t color_space,
                            uint8_t* rgba);

/* denoise_and_tonemap_frame_with_params_into: accum / spp, denoise with the given
 * guides (`path_sig` NULL: none), tone-map to sRGB RGBA8; spp == 0 gives opaque black. */
int ix_denoise_and_tonemap_frame(struct ix_backend* b, uint32_t width, uint32_t height,
                                 uint32_t spp, const float* accum, const float* depth,
                                 const float* normal, const int32_t* facet_id,
                                 const uint32_t* path_sig, const ix_atrous_params* params,
                                 uint8_t* rgba);

/* The display step of one accumulated frame, device-resident end to end: the guides of
 * `scene` (camera, planes; path signature at the material's n_d when `with_signature`)
 * computed on the device and cached for the next call with the same camera and planes,
 * then ix_denoise_and_tonemap_frame on them.  `accum` holds scene->width * height XYZ
 * sums as f32.  The result equals ix_generate_guide_buffers followed by
 * ix_denoise_and_tonemap_frame. */
int ix_display_frame(struct ix_backend* b, const ix_scene* scene, uint32_t with_signature,
                     uint32_t spp, const float* accum, const ix_atrous_params* params,
                     uint8_t* rgba);

/* Device-resident form of ix_display_frame (no counterpart in the reference): `accum` and
 * `rgba` are device pointers, scene->planes stays a host pointer (it keys the guide
 * cache); the kernels are enqueued on `stream` (a cudaStream_t, NULL for the backend's
 * own) and not synchronised.  With spp == 0 the frame is opaque black. */
int ix_display_frame_device(struct ix_backend* b, const ix_scene* scene, uint32_t with_signature,
                            uint32_t spp, const float* accum, const ix_atrous_params* params,
                            uint8_t* rgba, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IX_DISPLAY_H */
