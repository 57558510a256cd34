/*
 * ix_design.h -- parametric round-brilliant designs traced in batches: the design space
 * the learned surrogate (ix_surrogate.h) is trained over and that design search explores.
 *
 * A design is 12 numbers: the crown and pavilion main angles, the star, upper-half and
 * lower-half offsets from them, table and girdle sizes, the material's n_D and dispersion,
 * and one Gaussian absorption band.  ix_evaluate_designs builds each design's facet
 * half-spaces and material on the host, renders it at every requested view with the
 * batched path tracer (one persistent launch over designs x views, ix_batch_plan_*) as
 * two renders over disjoint halves a, b of the sample range, and reduces each view on the
 * device to three image metrics over the stone's pixels:
 *   brilliance     mean luminance Y (the environment's radiance is the unit);
 *   fire           RMS chromaticity offset from the equal-energy white, each pixel
 *                  weighted by S^2 (S = X + Y + Z): sqrt(sum N_a . N_b / sum S_a S_b) with
 *                  N = (X - S / 3, Y - S / 3) of one half;
 *   scintillation  spatial coefficient of variation of Y, sqrt(cov(Y_a, Y_b)) / mean Y.
 * Products of independent halves keep per-pixel sampling noise out of the two
 * second-moment metrics (one render's |N|^2 or var(Y) would grow with it), and no
 * per-pixel ratio is formed, so they converge with spp without a noise bias.  The stone's pixels are those whose primary ray
 * through the pixel centre enters the stone's half-space set.  These are measurements on the tracer's renders; they stand in
 * for, and are not, the reference's analytic metric estimators
 * (crates/indicatrix/src/color/metrics/evaluate.rs:158).
 *
 * No reference counterpart as an entry point: the reference's cut optimiser scores designs
 * with the analytic metrics (crates/indicatrix-cut-core/src/optimize/mod.rs:1-80).
 */
#ifndef IX_DESIGN_H
#define IX_DESIGN_H

#include <stdint.h>

#include "ix_cuda.h"
#include "ix_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

#define IX_DESIGN_PARAMS 12

typedef struct ix_design {
    float crown_deg;              /* crown main angle from the girdle plane             */
    float pavilion_deg;           /* pavilion main angle                                */
    float star_offset_deg;        /* star angle minus the crown angle                   */
    float upper_half_offset_deg;  /* upper girdle halves minus the crown angle          */
    float lower_half_offset_deg;  /* lower girdle halves minus the pavilion angle       */
    float table_pct;              /* table width, % of the girdle diameter              */
    float girdle_pct;             /* girdle thickness, % of the diameter                */
    float n_d;                    /* refractive index at 589.3 nm                       */
    float dispersion;             /* n(486.1 nm) - n(656.3 nm), Cauchy n = A + B / l^2  */
    float absorb_peak;            /* Gaussian band peak, 1/cm                           */
    float absorb_center_nm;       /* band centre                                        */
    float absorb_width_nm;        /* band width (the Gaussian's sigma)                  */
} ix_design;

/* What every design is traced under: one camera per view (a tilt), the environment, the
 * image size, the sample range (spp >= 2: the first spp / 2 samples are half a, the rest
 * half b) and the transport depth.  A girdle of girdle_segments
 * vertical planes (0: 64) closes the outline; the diameter is 1.0 and a model unit is
 * 0.65 cm for the absorption band. */
typedef struct ix_design_view {
    const ix_camera* cameras;
    uint32_t n_views;
    uint32_t width;
    uint32_t height;
    uint32_t spp;
    uint32_t sample_offset;
    uint32_t max_bounces;
    uint32_t girdle_segments;
    ix_environment environment;
} ix_design_view;

/* The design's facet half-spaces as f32 {nx, ny, nz, d} rows (n . x + d <= 0 inside):
 * table, stars, crown mains, upper halves, girdle, pavilion mains, lower halves.  Writes
 * at most `cap` planes; returns the count the design has (57 + girdle_segments: 1 + 8 +
 * 8 + 16 on the crown, 8 + 16 on the pavilion), or 0 when a parameter is out of its
 * domain. */
uint32_t ix_design_planes(const ix_design* d, uint32_t girdle_segments, float* planes, uint32_t cap);
/* The design's material: Cauchy dispersion through (n_D, dispersion), isotropic, with
 * the absorption band when absorb_peak > 0.  0 on success, -1 on a bad parameter. */
int ix_design_material(const ix_design* d, ix_material* out);

/* Traces designs x views in one batched launch and writes their metrics,
 * out[(i * n_views + v) * 3 + {0, 1, 2}] = brilliance, fire, scintillation of design i at
 * view v.  Returns IX_DONE, or IX_DECLINED (bad argument, a design out of its domain,
 * the device lost, or a launch error; ix_last_error says which). */
int ix_evaluate_designs(ix_backend* b, const ix_design* designs, uint32_t n, const ix_design_view* view,
                        float* out);

#ifdef __cplusplus
}
#endif

#endif /* IX_DESIGN_H */
