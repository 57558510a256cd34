"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (``libix_oracle.so``).

The oracle restates the reference's CPU spectral tracer in C++ (``ix_oracle.cpp``).  The
test suite, the smoke check and the benchmark's CPU-baseline leg load it as the checker
and as the reported CPU baseline; nothing in ``indicatrix_b200`` imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from indicatrix_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))


class PathInfo(C.Structure):
    _fields_ = [
        ("bounces", C.c_uint32),
        ("termination", C.c_uint32),
        ("escaped", C.c_uint32),
        ("exit_splits", C.c_uint32),
    ]


class PathEvents(C.Structure):
    """ixo_path_events: what one traced path did (transport/path_events.rs:27)."""

    _fields_ = [
        ("first_facet", C.c_int32),
        ("first_entered", C.c_uint32),
        ("exit_facet", C.c_int32),
        ("exit_normal", C.c_float * 3),
        ("exit_dir", C.c_float * 3),
        ("exit_bounce", C.c_uint32),
        ("bounces_before_exit", C.c_uint32),
        ("reentered", C.c_uint32),
        ("termination", C.c_uint32),
        ("has_escaped_dir", C.c_uint32),
        ("escaped_dir", C.c_float * 3),
        ("scattered", C.c_uint32),
    ]


TERM_ESCAPED, TERM_RR, TERM_CAP, TERM_SCATTER_ABSORBED = 0, 1, 2, 3


class FlopCounts(C.Structure):
    _fields_ = [
        ("add", C.c_uint64),
        ("mul", C.c_uint64),
        ("fma", C.c_uint64),
        ("div", C.c_uint64),
        ("sqrt", C.c_uint64),
        ("transcendental", C.c_uint64),
        ("paths", C.c_uint64),
    ]

    def flops(self) -> int:
        """Floating-point operations: add/sub, mul, div and sqrt count one, FMA two."""
        return int(self.add + self.mul + 2 * self.fma + self.div + self.sqrt)


def build() -> None:
    """Compile both oracle builds (plain and operation-counting) with make."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_LIBS: dict[str, C.CDLL] = {}


def _load(name: str) -> C.CDLL:
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P = C.POINTER
    f32p = P(C.c_float)
    lib.ixo_hash_u32.restype = C.c_uint32
    lib.ixo_hash_u32.argtypes = [C.c_uint32]
    lib.ixo_low_discrepancy_base2.restype = C.c_float
    lib.ixo_low_discrepancy_base2.argtypes = [C.c_uint32]
    lib.ixo_radical_inverse_base.restype = C.c_float
    lib.ixo_radical_inverse_base.argtypes = [C.c_uint32, C.c_uint32]
    lib.ixo_pixel_rotations.argtypes = [C.c_uint32, f32p]
    lib.ixo_sample_draws.argtypes = [C.c_uint32, C.c_uint32, f32p, P(C.c_uint32), f32p]
    lib.ixo_camera_new.argtypes = [C.c_float] * 4 + [P(abi.Camera)]
    lib.ixo_generate_ray.argtypes = [P(abi.Camera)] + [C.c_float] * 6 + [f32p, f32p]
    lib.ixo_hero_wavelengths.argtypes = [C.c_float, f32p]
    lib.ixo_dispersion_eval.restype = C.c_float
    lib.ixo_dispersion_eval.argtypes = [P(abi.Dispersion), C.c_float]
    lib.ixo_cmf.argtypes = [C.c_float, f32p]
    lib.ixo_d65.restype = C.c_float
    lib.ixo_d65.argtypes = [C.c_float]
    lib.ixo_exp_lane.restype = C.c_float
    lib.ixo_exp_lane.argtypes = [C.c_float]
    lib.ixo_tir_phase_delta.restype = C.c_float
    lib.ixo_tir_phase_delta.argtypes = [C.c_float] * 3
    lib.ixo_fresnel_reflect_apply.argtypes = [C.c_float, C.c_float, f32p, f32p]
    lib.ixo_intersect.restype = C.c_int
    lib.ixo_intersect.argtypes = [f32p, C.c_uint32, f32p, f32p, f32p, P(C.c_int32)]
    lib.ixo_environment_preset.restype = C.c_int
    lib.ixo_environment_preset.argtypes = [C.c_int32] + [C.c_float] * 6 + [P(abi.Environment)]
    lib.ixo_environment_uniform.argtypes = [C.c_float, P(abi.Environment)]
    lib.ixo_environment_channel.restype = C.c_float
    lib.ixo_environment_channel.argtypes = [P(abi.Environment), f32p, C.c_float, f32p]
    lib.ixo_trace_ray.restype = C.c_int
    lib.ixo_trace_ray.argtypes = [P(abi.Scene), f32p, f32p, C.c_uint32, C.c_float, f32p, P(PathInfo)]
    lib.ixo_trace_sample.restype = C.c_int
    lib.ixo_trace_sample.argtypes = [P(abi.Scene), C.c_uint32, C.c_uint32, f32p, P(PathInfo)]
    lib.ixo_trace_frame.restype = C.c_int64
    lib.ixo_trace_frame.argtypes = [P(abi.Scene), C.c_uint32, C.c_uint32, C.c_uint32, f32p,
                                    P(C.c_double)]
    lib.ixo_trace_pixels.restype = C.c_int64
    lib.ixo_trace_pixels.argtypes = [P(abi.Scene), C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.c_uint32, C.c_uint32, P(C.c_double)]
    lib.ixo_trace_samples.restype = C.c_int
    lib.ixo_trace_samples.argtypes = [P(abi.Scene), C.c_uint32, C.c_uint32, C.c_uint32,
                                      C.c_uint32, C.c_uint32, f32p, P(C.c_uint32)]
    lib.ixo_standard_round_brilliant.restype = C.c_uint32
    lib.ixo_standard_round_brilliant.argtypes = [f32p]
    lib.ixo_metrics.restype = C.c_int
    lib.ixo_metrics.argtypes = [f32p, C.c_uint32, P(abi.Material), C.c_float, C.c_float, C.c_int32,
                                C.c_float, C.c_float, C.c_float, f32p]
    lib.ixo_metrics_half_width.restype = C.c_float
    lib.ixo_metrics_half_width.argtypes = [f32p, C.c_uint32]
    lib.ixo_metrics_lighting.restype = C.c_int
    lib.ixo_metrics_lighting.argtypes = [C.c_int32, C.c_float, C.c_float, C.c_float, f32p]
    lib.ixo_trace_ray_events.restype = C.c_int
    lib.ixo_trace_ray_events.argtypes = [P(abi.Scene), f32p, f32p, C.c_uint32, C.c_float, f32p,
                                         P(PathEvents)]
    lib.ixo_path_events_reset.argtypes = [P(PathEvents)]
    lib.ixo_path_events_facet.argtypes = [P(PathEvents), C.c_uint32, C.c_int32, f32p, C.c_uint32, C.c_uint32,
                                          f32p]
    lib.ixo_classify_path.restype = C.c_int
    lib.ixo_classify_path.argtypes = [P(PathEvents), f32p, C.c_int32, C.c_float, C.c_float, C.c_float]
    lib.ixo_attribution_add.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float]
    lib.ixo_attribute_pixels.restype = C.c_int64
    lib.ixo_attribute_pixels.argtypes = [P(abi.Scene), C.c_int32, C.c_float, C.c_float, C.c_float,
                                         C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.c_void_p, P(C.c_double)]
    lib.ixo_trace_pixel_set.restype = C.c_int64
    lib.ixo_trace_pixel_set.argtypes = [P(abi.Scene), C.c_uint32, P(C.c_uint32), P(C.c_uint32), P(C.c_uint32),
                                        C.c_uint32, C.c_uint32, C.c_uint32, P(C.c_double)]
    lib.ixo_simd_build.restype = C.c_int
    lib.ixo_spectral_absorption.restype = C.c_float
    lib.ixo_spectral_absorption.argtypes = [P(abi.Absorption), C.c_float]
    lib.ixo_rotate_stokes.argtypes = [f32p, f32p, f32p, C.c_uint32, f32p, f32p, f32p]
    lib.ixo_fresnel_channel.argtypes = [C.c_float, C.c_float, C.c_float, f32p, f32p]
    lib.ixo_channel_alpha.restype = C.c_float
    lib.ixo_channel_alpha.argtypes = [P(abi.Material), f32p, C.c_float]
    lib.ixo_tool_ray_interval.restype = C.c_int
    lib.ixo_tool_ray_interval.argtypes = [P(abi.Tool), f32p, f32p, f32p]
    lib.ixo_tool_contains.restype = C.c_int
    lib.ixo_tool_contains.argtypes = [P(abi.Tool), f32p]
    lib.ixo_tool_boundary_gap.restype = C.c_float
    lib.ixo_tool_boundary_gap.argtypes = [P(abi.Tool), f32p]
    lib.ixo_tool_outward_normal.restype = None
    lib.ixo_tool_outward_normal.argtypes = [P(abi.Tool), f32p, f32p]
    lib.ixo_intersect_stone.restype = C.c_int
    lib.ixo_intersect_stone.argtypes = [f32p, C.c_uint32, P(abi.Tool), C.c_uint32, f32p, f32p, f32p, f32p,
                                        P(C.c_int32), P(C.c_int32)]
    lib.ixo_sun_nee_sample.restype = C.c_float
    lib.ixo_sun_nee_sample.argtypes = [P(abi.Environment), C.c_float, C.c_float, f32p]
    lib.ixo_sun_nee_pdf.restype = C.c_float
    lib.ixo_sun_nee_pdf.argtypes = [P(abi.Environment), f32p]
    lib.ixo_balance_heuristic.restype = C.c_float
    lib.ixo_balance_heuristic.argtypes = [C.c_float, C.c_float]
    lib.ixo_frosted_sun_nee.restype = None
    lib.ixo_frosted_sun_nee.argtypes = [P(abi.Scene), f32p, f32p, C.c_uint32, C.c_uint32, f32p, f32p, f32p]
    lib.ixo_biaxial_bundle.restype = None
    lib.ixo_biaxial_bundle.argtypes = [P(abi.Material), f32p, f32p, C.c_float, C.c_float, C.c_float, f32p]
    lib.ixo_counting_build.restype = C.c_int
    lib.ixo_count_flops.restype = C.c_int
    lib.ixo_count_flops.argtypes = [P(abi.Scene), C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.c_uint32, P(FlopCounts)]
    i32p, u32p, u8p = P(C.c_int32), P(C.c_uint32), P(C.c_uint8)
    lib.ixo_atrous_params_default.argtypes = [P(abi.AtrousParams)]
    lib.ixo_generate_guide_buffers.argtypes = [C.c_uint32, C.c_uint32, P(abi.Camera), f32p, C.c_uint32,
                                               C.c_float, f32p, f32p, i32p, u32p, C.c_int]
    lib.ixo_n_d.restype = C.c_float
    lib.ixo_n_d.argtypes = [P(abi.Dispersion)]
    lib.ixo_atrous_denoise.argtypes = [f32p, f32p, f32p, i32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32,
                                       P(abi.AtrousParams), f32p, C.c_int]
    lib.ixo_color_encode.argtypes = [f32p, C.c_uint32, u8p]
    lib.ixo_shading_normal_near_edge.argtypes = [f32p, C.c_uint32, f32p, C.c_int32, f32p, C.c_float, f32p]
    lib.ixo_count_denoise_flops.restype = C.c_int
    lib.ixo_count_denoise_flops.argtypes = [f32p, f32p, f32p, i32p, u32p, C.c_uint32, C.c_uint32, C.c_uint32,
                                            P(abi.AtrousParams), P(FlopCounts)]
    lib.ixo_tonemap_to_rgba.argtypes = [f32p, C.c_uint64, C.c_float, C.c_uint32, u8p, C.c_int]
    lib.ixo_denoise_and_tonemap_frame.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, f32p, f32p, f32p, i32p,
                                                  u32p, P(abi.AtrousParams), u8p, C.c_int]
    _LIBS[name] = lib
    return lib


def lib() -> C.CDLL:
    return _load("libix_oracle.so")


def counting_lib() -> C.CDLL:
    return _load("libix_oracle_count.so")


def host_has_avx2() -> bool:
    """True when this host's CPU reports AVX2 and FMA (the AVX2 build's instructions)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return "avx2" in flags and "fma" in flags
    except OSError:
        pass
    return False


def simd_lib() -> C.CDLL:
    """The AVX2 build (bit-identical to lib()) on hosts with AVX2 and FMA, else lib()."""
    return _load("libix_oracle_avx2.so") if host_has_avx2() else lib()


def trace_pixel_set(scenes, entries, sample_offset: int = 0, threads: int = 0, library=None, sums: bool = False):
    """Traces (scene index, pixel, spp) entries over ``scenes`` (abi.Scene list), claimed one
    at a time by ``threads`` host threads (0: all).  Returns (paths traced, dropped, per-entry
    f64 sums or None)."""
    if threads <= 0:
        threads = os.cpu_count() or 1
    library = library or lib()
    arr = (abi.Scene * len(scenes))(*scenes)
    e = np.ascontiguousarray(entries, np.uint32).reshape(-1, 3)
    cols = [np.ascontiguousarray(e[:, i]) for i in range(3)]
    out = np.zeros((e.shape[0], 3), np.float64) if sums else None
    u32p = C.POINTER(C.c_uint32)
    rc = library.ixo_trace_pixel_set(arr, len(scenes), cols[0].ctypes.data_as(u32p), cols[1].ctypes.data_as(u32p),
                                     cols[2].ctypes.data_as(u32p), e.shape[0], sample_offset, threads,
                                     out.ctypes.data_as(C.POINTER(C.c_double)) if sums else None)
    if rc < 0:
        raise ValueError("scene not supported by the oracle, or an entry out of range")
    return int(cols[2].astype(np.uint64).sum()), int(rc), out


def _f32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def sample_draws(pixel: int, sample: int, rot=None):
    out = np.zeros(3, np.float32)
    seed = C.c_uint32()
    r = None if rot is None else _f32p(np.asarray(rot, np.float32))
    lib().ixo_sample_draws(pixel, sample, r, C.byref(seed), _f32p(out))
    return int(seed.value), out


def pixel_rotations(pixel: int) -> np.ndarray:
    out = np.zeros(3, np.float32)
    lib().ixo_pixel_rotations(pixel, _f32p(out))
    return out


def camera_new(yaw: float, pitch: float, distance: float, fov_deg: float) -> abi.Camera:
    cam = abi.Camera()
    lib().ixo_camera_new(yaw, pitch, distance, fov_deg, C.byref(cam))
    return cam


def environment_preset(preset: int, exposure=1.0, yaw=0.0, pitch=0.0, backdrop=0.0,
                       glare=1.0, head_shadow_deg=16.0) -> abi.Environment:
    env = abi.Environment()
    rc = lib().ixo_environment_preset(preset, exposure, yaw, pitch, backdrop, glare,
                                      head_shadow_deg, C.byref(env))
    if rc != 0:
        raise ValueError(f"preset {preset} not modelled by the oracle")
    return env


def environment_uniform(radiance: float) -> abi.Environment:
    env = abi.Environment()
    lib().ixo_environment_uniform(radiance, C.byref(env))
    return env


def standard_round_brilliant() -> np.ndarray:
    out = np.zeros((74, 4), np.float32)
    n = lib().ixo_standard_round_brilliant(_f32p(out))
    assert n == 74
    return out


def trace_ray(scene: abi.Scene, origin, direction, seed: int, hero_rand: float):
    o = np.asarray(origin, np.float32)
    d = np.asarray(direction, np.float32)
    xyz = np.zeros(3, np.float32)
    info = PathInfo()
    rc = lib().ixo_trace_ray(C.byref(scene), _f32p(o), _f32p(d), seed, hero_rand, _f32p(xyz),
                             C.byref(info))
    if rc != 0:
        raise ValueError("scene not supported by the oracle")
    return xyz, info


def trace_sample(scene: abi.Scene, pixel: int, sample: int):
    xyz = np.zeros(3, np.float32)
    info = PathInfo()
    rc = lib().ixo_trace_sample(C.byref(scene), pixel, sample, _f32p(xyz), C.byref(info))
    if rc != 0:
        raise ValueError("scene not supported by the oracle")
    return xyz, info


def trace_frame(scene: abi.Scene, sample_offset: int, spp: int, threads: int = 0):
    """Returns (f32 sums [h, w, 3] in the reference's order, f64 sums, dropped count)."""
    if threads <= 0:
        threads = os.cpu_count() or 1
    n = scene.width * scene.height
    s32 = np.zeros((n, 3), np.float32)
    s64 = np.zeros((n, 3), np.float64)
    dropped = lib().ixo_trace_frame(C.byref(scene), sample_offset, spp, threads, _f32p(s32),
                                    s64.ctypes.data_as(C.POINTER(C.c_double)))
    if dropped < 0:
        raise ValueError("scene not supported by the oracle")
    return (s32.reshape(scene.height, scene.width, 3), s64.reshape(scene.height, scene.width, 3),
            int(dropped))


def trace_pixels(scene: abi.Scene, pixel_begin: int, pixel_end: int, sample_offset: int,
                 spp: int, threads: int = 0) -> np.ndarray:
    if threads <= 0:
        threads = os.cpu_count() or 1
    out = np.zeros((pixel_end - pixel_begin, 3), np.float64)
    rc = lib().ixo_trace_pixels(C.byref(scene), pixel_begin, pixel_end, sample_offset, spp,
                                threads, out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc < 0:
        raise ValueError("scene not supported by the oracle")
    return out


def trace_samples(scene: abi.Scene, pixel_begin: int, pixel_end: int, sample_offset: int,
                  spp: int, threads: int = 0):
    if threads <= 0:
        threads = os.cpu_count() or 1
    n = pixel_end - pixel_begin
    xyz = np.zeros((n, spp, 3), np.float32)
    bounces = np.zeros((n, spp), np.uint32)
    rc = lib().ixo_trace_samples(C.byref(scene), pixel_begin, pixel_end, sample_offset, spp,
                                 threads, _f32p(xyz),
                                 bounces.ctypes.data_as(C.POINTER(C.c_uint32)))
    if rc != 0:
        raise ValueError("scene not supported by the oracle")
    return xyz, bounces


def count_flops(scene: abi.Scene, pixel_begin: int, pixel_end: int, pixel_step: int,
                sample_offset: int, spp: int) -> FlopCounts:
    out = FlopCounts()
    rc = counting_lib().ixo_count_flops(C.byref(scene), pixel_begin, pixel_end, pixel_step,
                                        sample_offset, spp, C.byref(out))
    if rc != 0:
        raise ValueError("flop counting failed")
    return out


def metrics(planes: np.ndarray, material: abi.Material, cam_yaw: float, cam_pitch: float, preset: int,
            light_yaw: float, light_pitch: float, head_shadow_deg: float = 16.0) -> np.ndarray:
    """evaluate_gem_optical_metrics: [brilliance %, fire index, scintillation %,
    windowing %, extinction %] as float32."""
    p = np.ascontiguousarray(planes, np.float32)
    out = np.zeros(5, np.float32)
    rc = lib().ixo_metrics(_f32p(p), p.shape[0], C.byref(material), cam_yaw, cam_pitch, preset, light_yaw,
                           light_pitch, head_shadow_deg, _f32p(out))
    if rc != 0:
        raise ValueError("metrics: unmodelled preset or empty stone")
    return out


def metrics_half_width(planes: np.ndarray) -> float:
    p = np.ascontiguousarray(planes, np.float32)
    return float(lib().ixo_metrics_half_width(_f32p(p), p.shape[0]))


def metrics_lighting(preset: int, light_yaw: float, light_pitch: float, head_shadow_deg: float = 16.0):
    out = np.zeros(3, np.float32)
    if lib().ixo_metrics_lighting(preset, light_yaw, light_pitch, head_shadow_deg, _f32p(out)) != 0:
        raise ValueError("unmodelled preset")
    return out


def trace_ray_events(scene: abi.Scene, origin, direction, seed: int, hero_rand: float):
    """trace_spectral_ray_attributed_soa_geom: (xyz, PathEvents)."""
    o = np.asarray(origin, np.float32)
    d = np.asarray(direction, np.float32)
    xyz = np.zeros(3, np.float32)
    ev = PathEvents()
    rc = lib().ixo_trace_ray_events(C.byref(scene), _f32p(o), _f32p(d), seed, hero_rand, _f32p(xyz),
                                    C.byref(ev))
    if rc != 0:
        raise ValueError("scene not supported by the oracle")
    return xyz, ev


def classify_path(events: PathEvents, observer, preset: int, light_yaw: float, light_pitch: float,
                  head_shadow_deg: float = 16.0) -> int:
    """classify_path + class_index: the class slot, or abi.CLASS_MISS."""
    ob = np.asarray(observer, np.float32)
    r = lib().ixo_classify_path(C.byref(events), _f32p(ob), preset, light_yaw, light_pitch,
                                head_shadow_deg)
    if r < 0:
        raise ValueError("unmodelled preset")
    return int(r)


def attribution_add(pixel_map: np.ndarray, index: int, class_code: int, y: float,
                    scattered: bool = False, fluoresced: bool = False) -> None:
    """AttributionPixel::add on element `index` of a map (abi.attribution_dtype())."""
    assert pixel_map.dtype == abi.attribution_dtype() and pixel_map.flags.c_contiguous
    addr = pixel_map.ctypes.data + index * pixel_map.dtype.itemsize
    lib().ixo_attribution_add(C.c_void_p(addr), class_code, int(scattered), int(fluoresced), y)


def attribute_pixels(scene: abi.Scene, lighting: abi.MetricsLighting, pixel_begin: int, pixel_end: int,
                     sample_offset: int, spp: int, threads: int = 0, pixel_map=None, sums=None):
    """The attributed frame loop over pixels [pixel_begin, pixel_end): returns
    (map, f64 XYZ sums, dropped).  `pixel_map` / `sums` are accumulated when given."""
    if threads <= 0:
        threads = os.cpu_count() or 1
    n = pixel_end - pixel_begin
    if pixel_map is None:
        pixel_map = np.zeros(n, abi.attribution_dtype())
    if sums is None:
        sums = np.zeros((n, 3), np.float64)
    dropped = lib().ixo_attribute_pixels(C.byref(scene), lighting.preset, lighting.light_yaw,
                                         lighting.light_pitch, lighting.head_shadow_deg, pixel_begin,
                                         pixel_end, sample_offset, spp, threads,
                                         C.c_void_p(pixel_map.ctypes.data),
                                         sums.ctypes.data_as(C.POINTER(C.c_double)))
    if dropped < 0:
        raise ValueError("scene or lighting not supported by the oracle")
    return pixel_map, sums, int(dropped)


def path_events() -> PathEvents:
    """PathEvents::default."""
    ev = PathEvents()
    lib().ixo_path_events_reset(C.byref(ev))
    return ev


def path_events_facet(events: PathEvents, bounce: int, facet: int, normal, inside_before: bool,
                      inside_after: bool, dir_after) -> None:
    """PathEvents::facet for one facet event."""
    n = np.asarray(normal, np.float32)
    d = np.asarray(dir_after, np.float32)
    lib().ixo_path_events_facet(C.byref(events), bounce, facet, _f32p(n), int(inside_before), int(inside_after),
                                _f32p(d))


# ---- display pipeline (renderer/guide_pass.rs, renderer/denoise/, renderer/tonemap.rs) ----
def _ptr(a: np.ndarray, ctype):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def generate_guide_buffers(width: int, height: int, camera: abi.Camera, planes: np.ndarray, n_d: float = 0.0,
                           threads: int = 0):
    """generate_guide_buffers_with_index: (depth, normal[h, w, 3], facet_id, path_sig)."""
    planes = np.ascontiguousarray(planes, np.float32)
    depth = np.zeros((height, width), np.float32)
    normal = np.zeros((height, width, 3), np.float32)
    facet = np.zeros((height, width), np.int32)
    sig = np.zeros((height, width), np.uint32)
    lib().ixo_generate_guide_buffers(width, height, C.byref(camera), _f32p(planes), planes.shape[0], n_d,
                                     _f32p(depth), _f32p(normal), _ptr(facet, C.c_int32),
                                     _ptr(sig, C.c_uint32), threads)
    return depth, normal, facet, sig


def n_d(dispersion: abi.Dispersion) -> float:
    return float(lib().ixo_n_d(C.byref(dispersion)))


def atrous_denoise(color: np.ndarray, depth: np.ndarray, normal: np.ndarray, facet: np.ndarray, sig, spp: int,
                   params: abi.AtrousParams = None, threads: int = 0) -> np.ndarray:
    """AtrousDenoiser::denoise_into on [h, w, 3] float32 colour; `sig` None for no signature."""
    h, w = facet.shape
    params = params if params is not None else abi.AtrousParams.default()
    color = np.ascontiguousarray(color, np.float32)
    out = np.zeros((h, w, 3), np.float32)
    sig = None if sig is None else np.ascontiguousarray(sig, np.uint32)
    lib().ixo_atrous_denoise(_f32p(color), _f32p(np.ascontiguousarray(depth, np.float32)),
                             _f32p(np.ascontiguousarray(normal, np.float32)),
                             _ptr(np.ascontiguousarray(facet, np.int32), C.c_int32), _ptr(sig, C.c_uint32),
                             w, h, spp, C.byref(params), _f32p(out), threads)
    return out


def color_encode(xyz, color_space: int = abi.COLOR_SPACE_SRGB) -> bytes:
    """ColorSpace::encode with ToneMap::AcesFilmic { exposure: 1.0 }."""
    v = np.ascontiguousarray(xyz, np.float32)
    out = np.zeros(4, np.uint8)
    lib().ixo_color_encode(_f32p(v), color_space, _ptr(out, C.c_uint8))
    return bytes(out)


def tonemap_to_rgba(xyz: np.ndarray, scale: float = 1.0, color_space: int = abi.COLOR_SPACE_SRGB,
                    threads: int = 0) -> np.ndarray:
    """tonemap_to_rgba / tonemap_wide_gamut_with_threads: RGBA8 per pixel of `xyz` (..., 3)."""
    xyz = np.ascontiguousarray(xyz, np.float32)
    n = xyz.size // 3
    out = np.zeros(xyz.shape[:-1] + (4,), np.uint8)
    lib().ixo_tonemap_to_rgba(_f32p(xyz), n, scale, color_space, _ptr(out, C.c_uint8), threads)
    return out


def tonemap_accumulation(accum: np.ndarray, samples_per_pixel: int, color_space: int) -> np.ndarray:
    """tonemap_accumulation (tonemap.rs:213): encode(accum * (1 / spp)) in `color_space`."""
    inv = np.float32(1.0) / np.float32(samples_per_pixel)
    return tonemap_to_rgba(accum, float(inv), color_space)


def denoise_and_tonemap_frame(accum: np.ndarray, spp: int, depth, normal, facet, sig=None, params=None,
                              threads: int = 0) -> np.ndarray:
    """denoise_and_tonemap_frame_with_params_into: sRGB RGBA8 [h, w, 4]."""
    h, w = facet.shape
    params = params if params is not None else abi.AtrousParams.default()
    accum = np.ascontiguousarray(accum, np.float32)
    out = np.zeros((h, w, 4), np.uint8)
    sig = None if sig is None else np.ascontiguousarray(sig, np.uint32)
    lib().ixo_denoise_and_tonemap_frame(w, h, spp, _f32p(accum), _f32p(np.ascontiguousarray(depth, np.float32)),
                                        _f32p(np.ascontiguousarray(normal, np.float32)),
                                        _ptr(np.ascontiguousarray(facet, np.int32), C.c_int32),
                                        _ptr(sig, C.c_uint32), C.byref(params), _ptr(out, C.c_uint8), threads)
    return out


def count_denoise_flops(color, depth, normal, facet, sig, spp: int, params=None) -> FlopCounts:
    """Counting build: the operations of one A-Trous denoise; `paths` = pixel-passes."""
    h, w = facet.shape
    params = params if params is not None else abi.AtrousParams.default()
    out = FlopCounts()
    sig = None if sig is None else np.ascontiguousarray(sig, np.uint32)
    rc = counting_lib().ixo_count_denoise_flops(
        _f32p(np.ascontiguousarray(color, np.float32)), _f32p(np.ascontiguousarray(depth, np.float32)),
        _f32p(np.ascontiguousarray(normal, np.float32)), _ptr(np.ascontiguousarray(facet, np.int32), C.c_int32),
        _ptr(sig, C.c_uint32), w, h, spp, C.byref(params), C.byref(out))
    if rc != 0:
        raise RuntimeError("the counting oracle build is required")
    return out


def shading_normal_near_edge(planes: np.ndarray, hit_point, facet: int, hit_normal, radius: float) -> np.ndarray:
    planes = np.ascontiguousarray(planes, np.float32)
    out = np.zeros(3, np.float32)
    lib().ixo_shading_normal_near_edge(_f32p(planes), planes.shape[0], _f32p(np.asarray(hit_point, np.float32)),
                                       facet, _f32p(np.asarray(hit_normal, np.float32)), radius, _f32p(out))
    return out
