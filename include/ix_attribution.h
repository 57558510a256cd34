/*
 * ix_attribution.h -- the per-pixel spectral attribution record, shared by the CUDA
 * backend (libix_cuda.so) and every caller of its C ABI.
 *
 * One record per image pixel says what the pixel's path-traced samples did, by the
 * class `classify_path` (crates/indicatrix/src/color/metrics/attribution.rs:75) gives
 * each sample's hero path: a count per class and the luminance (the sample's XYZ.y)
 * the class delivered.  The layout and the update rule are the reference's
 * `AttributionPixel` (renderer/attribution_map.rs:80-120); the class slots are its
 * `CLASS_*` indices (attribution_map.rs:17-36) through `class_index` (:39-58).
 */
#ifndef IX_ATTRIBUTION_H
#define IX_ATTRIBUTION_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IX_ATTRIBUTION_CLASSES 9   /* ATTRIBUTION_CLASSES (attribution_map.rs:17)       */
#define IX_ATTRIBUTION_VERSION 1   /* SPECTRAL_ATTRIBUTION_VERSION (attribution.rs:19)  */
/* MAX_DIAGNOSTIC_PIXELS (color/metrics/image_types.rs:13): the largest map
 * AttributionMap::checked (attribution_map.rs:201) accepts. */
#define IX_ATTRIBUTION_MAX_PIXELS 1048576u

/* Class slots (attribution_map.rs:19-36). */
enum {
    IX_CLASS_GLARE = 0,           /* surface glare: the first facet event reflected outside */
    IX_CLASS_WINDOWED = 1,        /* first exit through a facet whose outward normal.y < -0.05 */
    IX_CLASS_RETURNED = 2,        /* first exit upward, outside the head shadow, towards a light */
    IX_CLASS_SHADOW = 3,          /* first exit upward into the observer's head shadow */
    IX_CLASS_UNLIT = 4,           /* first exit upward but not towards a light */
    IX_CLASS_SIDE_EXIT = 5,       /* first exit neither up (dir.y > 0.05) nor through the pavilion */
    IX_CLASS_NO_INTERSECTION = 6, /* entered, left the loop escaped without an exit event */
    IX_CLASS_BUDGET = 7,          /* entered, still inside when the bounce cap ran out */
    IX_CLASS_KILLED = 8           /* entered, ended by Russian roulette before an exit */
};
/* The class code of a camera ray that never met the stone (`classify_path` -> None). */
#define IX_CLASS_MISS 0xFF

/* AttributionPixel (attribution_map.rs:80-97), field for field. */
typedef struct ix_attribution_pixel {
    uint32_t samples;                         /* samples traced, misses included        */
    uint32_t hits;                            /* samples whose camera ray met the stone  */
    uint32_t counts[IX_ATTRIBUTION_CLASSES];  /* hits per class                          */
    float y_sum[IX_ATTRIBUTION_CLASSES];      /* delivered luminance per class (finite)  */
    float y_sq_sum[IX_ATTRIBUTION_CLASSES];   /* its square, for the standard error      */
    uint32_t scattered;                       /* hits whose path scattered               */
    uint32_t fluoresced;                      /* hits whose path fluoresced              */
} ix_attribution_pixel;

#ifdef __cplusplus
}
#endif

#endif /* IX_ATTRIBUTION_H */
