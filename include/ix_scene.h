/*
 * ix_scene.h -- plain-old-data scene description shared by the CUDA backend
 * (libix_cuda.so) and every caller of its C ABI.
 *
 * This is the C-ABI encoding of the reference's `GpuSceneRef`
 * (crates/indicatrix/src/renderer/gpu_backend/mod.rs:218-237): camera, image size,
 * facet half-space planes, per-facet finish, material, bounce cap and environment.
 * Field meanings follow the reference's GPU buffer layouts
 * (renderer/buffers/camera.rs:72-88, renderer/buffers/material.rs:93-243,
 * renderer/buffers/transport.rs:42-101) but the layout is this library's own:
 * everything a kernel needs per scene is resolved on the host into floats here, so a
 * device never evaluates a trig function of a light pose or camera pose.
 *
 * Units: model units for geometry (girdle diameter 1.0 for the generated cuts),
 * nanometres for wavelengths, and absorption coefficients in 1/length where
 * length = model units * absorption_path_scale.
 */
#ifndef IX_SCENE_H
#define IX_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IX_NUM_CHANNELS 8   /* hero-wavelength channels per path (transport/mod.rs:58) */
#define IX_MAX_PLANES 128   /* planes per stone the shared-memory cache holds          */
#define IX_MAX_BANDS 8      /* Gaussian bands per eigenmode (buffers/material.rs:93)     */
#define IX_SPLINE_KNOTS 16  /* knots of the tabulated absorption spline (new form)      */
#define IX_RING_LIGHTS 16   /* studio ring emitters (optics/studio_rig.rs:21)           */

/* Pinhole camera, the four vectors of `Camera` (optics/raytracer/camera.rs:89-101). */
typedef struct ix_camera {
    float origin[3];
    float forward[3];
    float right[3];
    float up[3];
    float fov_tan;
} ix_camera;

/* n(lambda) model (optics/dispersion.rs:4-9).
 *   IX_DISP_SELLMEIER1: b[0]=B1, c[0]=C1 (um^2)
 *   IX_DISP_SELLMEIER3: b[0..2], c[0..2]
 *   IX_DISP_CAUCHY:     b[0]=A, b[1]=B (um^2), b[2]=C (um^4)                        */
enum { IX_DISP_SELLMEIER1 = 0, IX_DISP_SELLMEIER3 = 1, IX_DISP_CAUCHY = 2 };
typedef struct ix_dispersion {
    uint32_t kind;
    float b[3];
    float c[3];
} ix_dispersion;

/* One absorption band (optics/absorption.rs:9-14). */
enum { IX_BAND_GAUSS_WAVELENGTH = 0, IX_BAND_GAUSS_ENERGY = 1 };
typedef struct ix_band {
    float center_nm;
    float width_nm;
    float peak;
    uint32_t shape;
} ix_band;

/* alpha(lambda) of one eigenmode: the sum of up to IX_MAX_BANDS Gaussian bands plus,
 * when has_spline != 0, a uniform Catmull-Rom spline through IX_SPLINE_KNOTS knots
 * spaced evenly over [380, 780] nm, floored at zero.  The spline is this library's
 * encoding of a smooth tabulated absorption curve; it has no reference counterpart. */
typedef struct ix_absorption {
    uint32_t n_bands;
    ix_band bands[IX_MAX_BANDS];
    uint32_t has_spline;
    float spline[IX_SPLINE_KNOTS];
} ix_absorption;

/* Material (GemMaterial, optics/materials/mod.rs:116-236, the fields the transport
 * reads).  `anisotropic` is the reference's `is_anisotropic`
 * (transport/inner.rs:191-193): crystal system not cubic and |birefringence_delta| > 1e-4. */
typedef struct ix_material {
    ix_dispersion dispersion;           /* ordinary index                            */
    uint32_t anisotropic;
    float birefringence_delta;          /* n_e - n_o for the walk-off approximation   */
    float c_axis[3];                    /* optic axis, unit length                    */
    uint32_t has_e_dispersion;          /* independent e-ray dispersion curve present */
    ix_dispersion e_dispersion;
    ix_absorption abs_o;                /* ordinary (isotropic: the only) absorption  */
    ix_absorption abs_e;                /* extraordinary absorption                   */
    float absorption_path_scale;        /* path length units per model unit           */
    float edge_rounding_radius;         /* 0 = sharp facet edges                      */
    float scattering_sigma_s;           /* Henyey-Greenstein interior scattering: sigma_s  */
                                        /* per model unit (0 = clear)                     */
    float scattering_g;                 /* HG asymmetry, -1 < g < 1                        */
    /* Biaxial indicatrix (GemMaterial::biaxial_indicatrix, materials/optics.rs:16): when
     * `biaxial` != 0, n_beta = dispersion(lambda), n_alpha = n_beta -
     * biaxial_delta_beta_alpha, n_gamma = n_alpha + birefringence_delta, with the gamma
     * axis along c_axis (BiaxialIndicatrix::from_gamma_axis, birefringence/biaxial.rs:58).
     * A biaxial material must also be `anisotropic`.  abs_o / abs_beta / abs_e are the
     * alpha / beta / gamma ray absorption (AbsorptionTensor::biaxial, absorption.rs:338);
     * without abs_beta the beta axis takes the alpha-ray value (the uniaxial tensor). */
    uint32_t biaxial;
    float biaxial_delta_beta_alpha;
    uint32_t has_abs_beta;
    ix_absorption abs_beta;
} ix_material;

/* Lighting model ids: the reference's LightingModel::gpu_id (environment/mod.rs:281-289)
 * plus a uniform furnace dome. */
enum {
    IX_ENV_STUDIO = 0,
    IX_ENV_ISO_HEMISPHERE = 1,
    IX_ENV_LIGHT_TENT = 2,
    IX_ENV_DAYLIGHT_DOME = 3,
    IX_ENV_ASET = 4,
    IX_ENV_DAYLIGHT_SUN = 5,
    IX_ENV_UNIFORM = 100
};
/* Illuminant spectral power (environment/spectral.rs:89-145): D65, a normalised blackbody,
 * flat, a Gaussian line (the UV lamps), and the wavelength itself (the ASET view's zone
 * bands read it, rig.rs:580). */
enum { IX_SPEC_D65 = 0, IX_SPEC_BLACKBODY = 1, IX_SPEC_FLAT = 2, IX_SPEC_GAUSSIAN = 3, IX_SPEC_WAVELENGTH = 4 };

typedef struct ix_environment {
    uint32_t model;
    uint32_t spectrum;
    float exposure;
    float spot_mult;            /* studio rig key/ring multiplier                       */
    uint32_t ambient_fill;      /* studio rig charcoal backdrop term present            */
    float backdrop;             /* lit tray below the horizon; 0 = none                 */
    float surface_glare;        /* first-bounce specular scale, clamped to [0, 1]        */
    float shadow_cos[2];        /* head-shadow smoothstep edges (environment/mod.rs:128) */
    float bb_t_k;               /* blackbody temperature (max(T, 1000))                  */
    float bb_denom_560;         /* blackbody normalisation at 560 nm                    */
    float key_dir[3];           /* StudioRig (optics/studio_rig.rs:33-70)                */
    float fill_dir[3];
    float ring_dirs[IX_RING_LIGHTS][3];
    uint32_t white_balance;     /* apply the Bradford von Kries round trip at finish     */
    float wb_lms[3];            /* LMS scale of the white balance                       */
    float uniform_radiance;     /* IX_ENV_UNIFORM dome radiance                         */
    /* TentParams (environment/mod.rs:185) of the IX_ENV_LIGHT_TENT presets. */
    float tent_walls, tent_cards, tent_spark, tent_ground, tent_flat;
    float sun_factor;           /* IX_ENV_DAYLIGHT_SUN: SUN_RADIANCE x horizon_blend(key_dir) */
    float line_centre_nm;       /* IX_SPEC_GAUSSIAN: line centre and sigma                  */
    float line_sigma_nm;
} ix_environment;

struct ix_tool;

/* The scene.  `planes` is n_planes x {nx, ny, nz, d} with the convention n.x + d <= 0
 * inside (geometry/plane.rs:34-41).  `facet_finishes` may be NULL (all polished); entry
 * i is facet i's FacetFinish (0 Polished, nonzero Frosted), facets past n_finishes are
 * polished. */
typedef struct ix_scene {
    ix_camera camera;
    uint32_t width;
    uint32_t height;
    const float* planes;
    uint32_t n_planes;
    const uint8_t* facet_finishes;
    uint32_t n_finishes;
    ix_material material;
    uint32_t max_bounces;
    ix_environment environment;
    /* Concave tools carved out of the stone (StoneGeometry::tools, geometry/tool.rs:173):
     * NULL / 0 for a convex stone.  Tool k has facet id n_planes + k.  The accumulate
     * entries take their `tools` / `ntools` arguments instead when ntools > 0. */
    const struct ix_tool* tools;
    uint32_t n_tools;
} ix_scene;

/* A concave tool volume subtracted from the stone (ToolPrimitive,
 * crates/indicatrix/src/geometry/tool.rs:112-131), field for field: the same 80-byte
 * record (the reference aligns it to 16 bytes): kind 0 ball, 1 capped cylinder, 2 cone
 * frustum, 3 bicone; sweep_kind 0 none, 1 along the axis, 2 across it.  At most
 * IX_MAX_TOOLS per stone (GPU_MAX_TOOL_PRIMITIVES, tool/pack.rs:51); a tool that fails
 * ToolPrimitive::validate (tool.rs:360) makes the scene decline. */
#define IX_MAX_TOOLS 128
typedef struct ix_tool {
    uint32_t kind;
    uint32_t sweep_kind;
    uint32_t pad[2];           /* zero                                                  */
    float origin[4];           /* centre xyz; w = radius at the centre                  */
    float axis[4];             /* unit axis xyz; w = half-length along it (0: a ball)   */
    float profile[4];          /* radius at -half_length, at +half_length, half-stroke, 0 */
    float sweep_dir[4];        /* unit sweep direction (sweep_kind 2), w = 0            */
} ix_tool;

#ifdef __cplusplus
}
#endif

#endif /* IX_SCENE_H */
