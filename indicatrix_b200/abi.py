"""ctypes mirror of ``include/ix_scene.h`` and ``include/ix_cuda.h``.

These structures are the C-ABI encoding of the reference's ``GpuSceneRef``
(crates/indicatrix/src/renderer/gpu_backend/mod.rs:218-237) and of the backend's
options, batch items and status codes.  Every field matches the C header one for one;
``tests/test_host.py`` checks sizes and offsets against the C headers.
"""
from __future__ import annotations

import ctypes as C

NUM_CHANNELS = 8
MAX_PLANES = 128
MAX_BANDS = 8
SPLINE_KNOTS = 16
RING_LIGHTS = 16
MAX_TOOLS = 128

DISP_SELLMEIER1, DISP_SELLMEIER3, DISP_CAUCHY = 0, 1, 2
BAND_GAUSS_WAVELENGTH, BAND_GAUSS_ENERGY = 0, 1
ENV_STUDIO, ENV_ISO_HEMISPHERE, ENV_UNIFORM = 0, 1, 100
ENV_LIGHT_TENT, ENV_DAYLIGHT_DOME, ENV_ASET, ENV_DAYLIGHT_SUN = 2, 3, 4, 5
SPEC_D65, SPEC_BLACKBODY, SPEC_FLAT, SPEC_GAUSSIAN, SPEC_WAVELENGTH = 0, 1, 2, 3, 4

# GpuAccumulate (gpu_backend/mod.rs:308-326) plus the internal error the C ABI maps to
# a decline.
IX_DONE, IX_DECLINED, IX_CANCELLED = 0, 1, 2

# GpuPipelineKind (gpu_backend/mod.rs:347-353).
PIPELINE_MEGAKERNEL, PIPELINE_WAVEFRONT = 0, 1
# Rounding modes of the transport kernels.
PRECISION_FAST, PRECISION_EXACT = 0, 1


class Camera(C.Structure):
    _fields_ = [
        ("origin", C.c_float * 3),
        ("forward", C.c_float * 3),
        ("right", C.c_float * 3),
        ("up", C.c_float * 3),
        ("fov_tan", C.c_float),
    ]


class Dispersion(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("b", C.c_float * 3), ("c", C.c_float * 3)]


class Band(C.Structure):
    _fields_ = [
        ("center_nm", C.c_float),
        ("width_nm", C.c_float),
        ("peak", C.c_float),
        ("shape", C.c_uint32),
    ]


class Absorption(C.Structure):
    _fields_ = [
        ("n_bands", C.c_uint32),
        ("bands", Band * MAX_BANDS),
        ("has_spline", C.c_uint32),
        ("spline", C.c_float * SPLINE_KNOTS),
    ]


class Material(C.Structure):
    _fields_ = [
        ("dispersion", Dispersion),
        ("anisotropic", C.c_uint32),
        ("birefringence_delta", C.c_float),
        ("c_axis", C.c_float * 3),
        ("has_e_dispersion", C.c_uint32),
        ("e_dispersion", Dispersion),
        ("abs_o", Absorption),
        ("abs_e", Absorption),
        ("absorption_path_scale", C.c_float),
        ("edge_rounding_radius", C.c_float),
        ("scattering_sigma_s", C.c_float),
        ("scattering_g", C.c_float),
        ("biaxial", C.c_uint32),
        ("biaxial_delta_beta_alpha", C.c_float),
        ("has_abs_beta", C.c_uint32),
        ("abs_beta", Absorption),
    ]


class Environment(C.Structure):
    _fields_ = [
        ("model", C.c_uint32),
        ("spectrum", C.c_uint32),
        ("exposure", C.c_float),
        ("spot_mult", C.c_float),
        ("ambient_fill", C.c_uint32),
        ("backdrop", C.c_float),
        ("surface_glare", C.c_float),
        ("shadow_cos", C.c_float * 2),
        ("bb_t_k", C.c_float),
        ("bb_denom_560", C.c_float),
        ("key_dir", C.c_float * 3),
        ("fill_dir", C.c_float * 3),
        ("ring_dirs", (C.c_float * 3) * RING_LIGHTS),
        ("white_balance", C.c_uint32),
        ("wb_lms", C.c_float * 3),
        ("uniform_radiance", C.c_float),
        ("tent_walls", C.c_float),
        ("tent_cards", C.c_float),
        ("tent_spark", C.c_float),
        ("tent_ground", C.c_float),
        ("tent_flat", C.c_float),
        ("sun_factor", C.c_float),
        ("line_centre_nm", C.c_float),
        ("line_sigma_nm", C.c_float),
    ]


class Tool(C.Structure):
    """ix_tool: a concave tool volume (ToolPrimitive, geometry/tool.rs:112), 80 bytes."""

    _fields_ = [
        ("kind", C.c_uint32),
        ("sweep_kind", C.c_uint32),
        ("pad", C.c_uint32 * 2),
        ("origin", C.c_float * 4),
        ("axis", C.c_float * 4),
        ("profile", C.c_float * 4),
        ("sweep_dir", C.c_float * 4),
    ]


class Scene(C.Structure):
    _fields_ = [
        ("camera", Camera),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("planes", C.POINTER(C.c_float)),
        ("n_planes", C.c_uint32),
        ("facet_finishes", C.POINTER(C.c_uint8)),
        ("n_finishes", C.c_uint32),
        ("material", Material),
        ("max_bounces", C.c_uint32),
        ("environment", Environment),
        ("tools", C.POINTER(Tool)),
        ("n_tools", C.c_uint32),
    ]


class BackendOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("pipeline", C.c_uint32),
        ("precision", C.c_uint32),
        ("threads_per_block", C.c_uint32),
        ("chunk_paths", C.c_uint64),
        ("kernel_variant", C.c_uint32),
    ]


class WorkLimits(C.Structure):
    _fields_ = [
        ("max_pixels", C.c_uint64),
        ("max_paths_per_call", C.c_uint64),
        ("max_spp", C.c_uint32),
    ]


# ix_batch_done_fn: on_done(user, index, status).
BATCH_DONE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_int32)


class BatchItem(C.Structure):
    """One stone of a batched launch (GpuBatchItem, gpu_backend/mod.rs:246)."""

    _fields_ = [
        ("scene", C.POINTER(Scene)),
        ("sample_offset", C.c_uint32),
        ("spp", C.c_uint32),
        ("accum_xyz", C.POINTER(C.c_double)),
        ("status", C.c_int32),
    ]


class BatchJob(C.Structure):
    """One job of a batch plan: a whole frame of one scene over an absolute sample range."""

    _fields_ = [
        ("scene", C.c_uint32),
        ("sample_offset", C.c_uint32),
        ("spp", C.c_uint32),
    ]


class TimingInfo(C.Structure):
    _fields_ = [
        ("kernel_ms", C.c_float),
        ("reduce_ms", C.c_float),
        ("paths", C.c_uint64),
        ("launches", C.c_uint32),
    ]


class GemMetrics(C.Structure):
    """GemOpticalMetrics (color/metrics/types.rs)."""

    _fields_ = [
        ("brilliance_pct", C.c_float),
        ("fire_index", C.c_float),
        ("scintillation_pct", C.c_float),
        ("windowing_pct", C.c_float),
        ("extinction_pct", C.c_float),
    ]


class MetricsLighting(C.Structure):
    _fields_ = [
        ("preset", C.c_int32),
        ("light_yaw", C.c_float),
        ("light_pitch", C.c_float),
        ("head_shadow_deg", C.c_float),
    ]


# Tilt-performance sweeps (include/ix_cuda.h): PROFILE_ANGLES_DEG (color/metrics/types.rs:27),
# TILT_ANGLES_DEG (profile.rs:146) and PROFILE_AZIMUTHS_DEG (profile.rs:26).
PROFILE_ANGLES = 19
AXIS_TILTS = 181
PROFILE_ANGLES_DEG = [5.0 * i for i in range(PROFILE_ANGLES)]
TILT_ANGLES_DEG = [float(i - 90) for i in range(AXIS_TILTS)]
PROFILE_AZIMUTHS_DEG = [0.0, 45.0, 90.0, 135.0]

# Spectral attribution (include/ix_attribution.h): the class slots of
# renderer/attribution_map.rs:17-36 and the code of a camera ray that missed the stone.
ATTRIBUTION_CLASSES = 9
ATTRIBUTION_VERSION = 1
(CLASS_GLARE, CLASS_WINDOWED, CLASS_RETURNED, CLASS_SHADOW, CLASS_UNLIT, CLASS_SIDE_EXIT,
 CLASS_NO_INTERSECTION, CLASS_BUDGET, CLASS_KILLED) = range(9)
CLASS_MISS = 0xFF


class AttributionPixel(C.Structure):
    """AttributionPixel (renderer/attribution_map.rs:80-97), field for field."""

    _fields_ = [
        ("samples", C.c_uint32),
        ("hits", C.c_uint32),
        ("counts", C.c_uint32 * ATTRIBUTION_CLASSES),
        ("y_sum", C.c_float * ATTRIBUTION_CLASSES),
        ("y_sq_sum", C.c_float * ATTRIBUTION_CLASSES),
        ("scattered", C.c_uint32),
        ("fluoresced", C.c_uint32),
    ]


def attribution_dtype():
    """The numpy structured dtype of ``ix_attribution_pixel`` (a map is an array of it)."""
    import numpy as np

    dt = np.dtype([
        ("samples", "<u4"),
        ("hits", "<u4"),
        ("counts", "<u4", (ATTRIBUTION_CLASSES,)),
        ("y_sum", "<f4", (ATTRIBUTION_CLASSES,)),
        ("y_sq_sum", "<f4", (ATTRIBUTION_CLASSES,)),
        ("scattered", "<u4"),
        ("fluoresced", "<u4"),
    ])
    assert dt.itemsize == C.sizeof(AttributionPixel)
    return dt


class MetricsStone(C.Structure):
    _fields_ = [
        ("planes", C.POINTER(C.c_float)),
        ("n_planes", C.c_uint32),
        ("dispersion", Dispersion),
    ]


class MetricsPose(C.Structure):
    _fields_ = [
        ("stone", C.c_uint32),
        ("cam_yaw", C.c_float),
        ("cam_pitch", C.c_float),
    ]


class AtrousParams(C.Structure):
    """ix_atrous_params (include/ix_display.h): AtrousParams, denoise/mod.rs:157."""

    _fields_ = [
        ("num_passes", C.c_uint32),
        ("sigma_color", C.c_float),
        ("sigma_depth", C.c_float),
        ("normal_power", C.c_float),
        ("taper_reference_spp", C.c_float),
        ("taper_identity_epsilon", C.c_float),
    ]

    @classmethod
    def default(cls) -> "AtrousParams":
        """AtrousParams::default (denoise/mod.rs:194)."""
        return cls(5, 0.35, 0.1, 64.0, 4.0, 0.02)


COLOR_SPACE_SRGB, COLOR_SPACE_DISPLAY_P3, COLOR_SPACE_REC2020, COLOR_SPACE_ACESCG = 0, 1, 2, 3


def floats(values) -> C.Array:
    arr = (C.c_float * len(values))()
    for i, v in enumerate(values):
        arr[i] = float(v)
    return arr
