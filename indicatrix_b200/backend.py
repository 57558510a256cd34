"""Host-side mirror of the reference's ``GpuBackend`` over ``libix_cuda.so``.

Same operation names, argument meaning and outcomes as
crates/indicatrix/src/renderer/gpu_backend/backend.rs (and its always-decline stub,
gpu_backend/stub.rs:12-138):

* ``GpuBackend.acquire()`` / ``GpuBackend.disabled()`` -- a usable backend or one that
  declines everything;
* ``try_accumulate(scene, sample_offset, spp, accum) -> bool`` -- adds the per-pixel sums
  of samples ``[sample_offset, sample_offset + spp)`` into ``accum`` (row-major
  ``height x width x 3``) and returns True, or returns False with ``accum`` untouched;
* ``try_accumulate_cancellable(...) -> GpuAccumulate`` -- DONE / DECLINED / CANCELLED;
* ``try_accumulate_batch_cancellable(items, cancel, on_done)``;
* ``is_lost`` / ``try_recover`` / ``adapter_label`` / ``set_pipeline_kind`` /
  ``set_work_limits``.

The CUDA library is the only compute path: if it is missing or fails to load, the
import raises; nothing here falls back to a CPU tracer.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
import threading
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libix_cuda.so")

_lib: Optional[C.CDLL] = None
_lib_lock = threading.Lock()


def load_library() -> C.CDLL:
    """Load ``libix_cuda.so`` (building it first if it is absent).  Raises on failure."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from .build import build

            build()
        lib = C.CDLL(LIB_PATH)
        P = C.POINTER
        lib.ix_backend_create.restype = C.c_void_p
        lib.ix_backend_create.argtypes = [P(abi.BackendOptions)]
        lib.ix_backend_destroy.argtypes = [C.c_void_p]
        lib.ix_backend_label.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        lib.ix_set_pipeline_kind.argtypes = [C.c_void_p, C.c_uint32]
        lib.ix_set_work_limits.argtypes = [C.c_void_p, P(abi.WorkLimits)]
        lib.ix_set_precision.argtypes = [C.c_void_p, C.c_uint32]
        lib.ix_scene_routes_to_gpu.argtypes = [P(abi.Scene)]
        lib.ix_scene_routes_to_gpu_with_tools.argtypes = [P(abi.Scene), P(abi.Tool), C.c_uint32]
        lib.ix_tool_validate.argtypes = [P(abi.Tool)]
        lib.ix_tool_validate.restype = C.c_int
        lib.ix_accumulate.argtypes = [C.c_void_p, P(abi.Scene), P(abi.Tool), C.c_uint32, C.c_uint32, C.c_uint32,
                                      P(C.c_float), P(C.c_uint8)]
        lib.ix_accumulate_f64.argtypes = [C.c_void_p, P(abi.Scene), P(abi.Tool), C.c_uint32, C.c_uint32,
                                          C.c_uint32, P(C.c_double), P(C.c_uint8)]
        lib.ix_accumulate_batch.argtypes = [C.c_void_p, P(abi.BatchItem), C.c_uint32, P(C.c_uint8),
                                            abi.BATCH_DONE_FN, C.c_void_p]
        lib.ix_accumulate_device.argtypes = [C.c_void_p, P(abi.Scene), C.c_uint32, C.c_uint32,
                                             C.c_void_p, C.c_int, C.c_void_p]
        lib.ix_is_lost.argtypes = [C.c_void_p]
        lib.ix_try_recover.argtypes = [C.c_void_p]
        lib.ix_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        lib.ix_last_timing.argtypes = [C.c_void_p, P(abi.TimingInfo)]
        lib.ix_last_dropped.restype = C.c_uint64
        lib.ix_last_dropped.argtypes = [C.c_void_p]
        lib.ix_probe_fp32_peak.argtypes = [C.c_void_p, P(C.c_double)]
        lib.ix_batch_plan_create.restype = C.c_void_p
        lib.ix_batch_plan_create.argtypes = [C.c_void_p, P(abi.Scene), C.c_uint32, P(abi.BatchJob),
                                             C.c_uint32]
        lib.ix_batch_plan_run.argtypes = [C.c_void_p, C.c_void_p]
        lib.ix_batch_plan_autotune.argtypes = [C.c_void_p, C.c_int, P(C.c_uint32)]
        lib.ix_batch_plan_set_variant.argtypes = [C.c_void_p, C.c_uint32]
        lib.ix_batch_plan_download.argtypes = [C.c_void_p, P(C.c_double)]
        lib.ix_batch_plan_output_size.restype = C.c_uint64
        lib.ix_batch_plan_output_size.argtypes = [C.c_void_p]
        lib.ix_batch_plan_device_output.restype = C.c_void_p
        lib.ix_batch_plan_device_output.argtypes = [C.c_void_p]
        lib.ix_batch_plan_paths.restype = C.c_uint64
        lib.ix_batch_plan_paths.argtypes = [C.c_void_p]
        lib.ix_batch_plan_variant.restype = C.c_uint32
        lib.ix_batch_plan_variant.argtypes = [C.c_void_p]
        lib.ix_batch_plan_job_offset.restype = C.c_uint64
        lib.ix_batch_plan_job_offset.argtypes = [C.c_void_p, C.c_uint32]
        lib.ix_batch_plan_destroy.argtypes = [C.c_void_p]
        lib.ix_camera_new.argtypes = [C.c_float] * 4 + [P(abi.Camera)]
        lib.ix_environment_preset.argtypes = [C.c_int32] + [C.c_float] * 6 + [P(abi.Environment)]
        lib.ix_environment_uniform.argtypes = [C.c_float, P(abi.Environment)]
        lib.ix_debug_check.argtypes = [C.c_void_p, P(abi.Scene), C.c_int32, C.c_uint32,
                                       P(C.c_uint32), C.c_uint32, P(C.c_uint32), C.c_uint32]
        lib.ix_evaluate_gem_optical_metrics.argtypes = [C.c_void_p, P(C.c_float), C.c_uint32, P(abi.Material),
                                                        C.c_float, C.c_float, P(abi.MetricsLighting),
                                                        P(abi.GemMetrics)]
        lib.ix_evaluate_gem_optical_metrics_batch.argtypes = [C.c_void_p, P(abi.MetricsStone), C.c_uint32,
                                                              P(abi.MetricsLighting), P(abi.MetricsPose),
                                                              C.c_uint32, C.c_uint32, P(abi.GemMetrics)]
        lib.ix_evaluate_angular_profile_at_azimuth.argtypes = [C.c_void_p, P(C.c_float), C.c_uint32,
                                                               P(abi.Material), C.c_float,
                                                               P(abi.MetricsLighting), P(C.c_float)]
        lib.ix_evaluate_axis_profiles.argtypes = [C.c_void_p, P(C.c_float), C.c_uint32, P(abi.Material),
                                                  P(C.c_float), C.c_uint32, P(abi.MetricsLighting),
                                                  P(C.c_float)]
        lib.ix_accumulate_attributed.argtypes = [C.c_void_p, P(abi.Scene), P(abi.MetricsLighting), C.c_uint32,
                                                 C.c_uint32, P(C.c_double), C.c_void_p, P(C.c_uint8)]
        _lib = lib
        return lib


class GpuAccumulate(enum.IntEnum):
    """Outcome of an accumulate call (gpu_backend/mod.rs:308-326)."""

    DONE = abi.IX_DONE
    DECLINED = abi.IX_DECLINED
    CANCELLED = abi.IX_CANCELLED


class GpuPipelineKind(enum.IntEnum):
    """gpu_backend/mod.rs:347-353."""

    MEGAKERNEL = abi.PIPELINE_MEGAKERNEL
    WAVEFRONT = abi.PIPELINE_WAVEFRONT


@dataclass
class GpuWorkLimits:
    """gpu_backend/limits.rs:6-27; zero means unlimited."""

    max_pixels: int = 0
    max_paths_per_call: int = 0
    max_spp: int = 0


class CancelFlag:
    """An ``AtomicBool``-like one-byte cancel flag the library polls between chunks."""

    def __init__(self) -> None:
        self._word = C.c_uint8(0)

    def set(self) -> None:
        self._word.value = 1

    def clear(self) -> None:
        self._word.value = 0

    def is_set(self) -> bool:
        return bool(self._word.value)

    def pointer(self):
        return C.pointer(self._word)


@dataclass
class FrameScene:
    """What a frame tracer needs (renderer/frame_scene.rs:22 / GpuSceneRef): the camera,
    image size, facet planes (n.x + d <= 0 inside), per-facet finishes, material, bounce
    cap and environment.  ``to_abi`` produces the C POD, keeping the arrays alive."""

    camera: abi.Camera
    width: int
    height: int
    planes: np.ndarray
    material: abi.Material
    max_bounces: int
    environment: abi.Environment
    facet_finishes: Optional[np.ndarray] = None
    tools: Optional[Sequence[abi.Tool]] = None  # concave tools; tool k is facet n_planes + k
    _keep: list = field(default_factory=list, repr=False)

    def to_abi(self) -> abi.Scene:
        planes = np.ascontiguousarray(self.planes, dtype=np.float32).reshape(-1, 4)
        sc = abi.Scene()
        sc.camera = self.camera
        sc.width = int(self.width)
        sc.height = int(self.height)
        sc.planes = planes.ctypes.data_as(C.POINTER(C.c_float))
        sc.n_planes = planes.shape[0]
        if self.facet_finishes is not None:
            fin = np.ascontiguousarray(self.facet_finishes, dtype=np.uint8)
            sc.facet_finishes = fin.ctypes.data_as(C.POINTER(C.c_uint8))
            sc.n_finishes = fin.shape[0]
            self._keep.append(fin)
        sc.material = self.material
        sc.max_bounces = int(self.max_bounces)
        sc.environment = self.environment
        if self.tools:
            arr = (abi.Tool * len(self.tools))(*self.tools)
            sc.tools = C.cast(arr, C.POINTER(abi.Tool))
            sc.n_tools = len(self.tools)
            self._keep.append(arr)
        self._keep.append(planes)
        return sc


def camera_new(yaw: float, pitch: float, distance: float, fov_deg: float = 42.0) -> abi.Camera:
    """Camera::new (optics/raytracer/camera.rs:108); DEFAULT_FOV_DEG is 42 (:66)."""
    cam = abi.Camera()
    load_library().ix_camera_new(yaw, pitch, distance, fov_deg, C.byref(cam))
    return cam


# LightingPreset::index (environment/mod.rs:475-493) for the presets this backend models.
PRESET_ISO_HEMISPHERE = 1
PRESET_DAYLIGHT = 7
PRESET_INCANDESCENT = 8
PRESET_ILLUMINANT_A = 9
PRESET_RING_LIGHTS = 10
PRESET_DARK_SPOTLIGHT = 11


def environment_preset(preset: int, exposure: float = 1.0, light_yaw: float = 0.0,
                       light_pitch: float = 0.0, backdrop: float = 0.0,
                       surface_glare: float = 1.0, head_shadow_deg: float = 16.0) -> abi.Environment:
    """EnvironmentSource::Studio { preset, .. } with its host-side derived fields."""
    env = abi.Environment()
    rc = load_library().ix_environment_preset(preset, exposure, light_yaw, light_pitch, backdrop,
                                              surface_glare, head_shadow_deg, C.byref(env))
    if rc != 0:
        raise ValueError(f"lighting preset {preset} is not modelled by this backend")
    return env


def environment_uniform(radiance: float) -> abi.Environment:
    env = abi.Environment()
    load_library().ix_environment_uniform(radiance, C.byref(env))
    return env


def scene_routes_to_gpu(scene: FrameScene) -> bool:
    """scene_routes_to_gpu (gpu_backend/mod.rs:288)."""
    return bool(load_library().ix_scene_routes_to_gpu(C.byref(scene.to_abi())))


def scene_routes_to_gpu_with_tools(scene: FrameScene, tools: Sequence[abi.Tool]) -> bool:
    """scene_routes_to_gpu_with_tools (gpu_backend/tool_routing.rs:81): any concave tool
    declines (this backend traces convex stones)."""
    tarr = (abi.Tool * len(tools))(*tools) if tools else None
    return bool(load_library().ix_scene_routes_to_gpu_with_tools(C.byref(scene.to_abi()), tarr, len(tools)))


# ToolPrimitiveError (geometry/tool.rs:133) as ix_tool_validate returns it.
TOOL_ERRORS = {0: None, 1: "NonFinite", 2: "NonPositiveRadius", 3: "AxisNotUnit", 4: "UnknownKind",
               5: "UnknownSweep", 6: "PaddingNotZero"}


def tool_validate(tool: abi.Tool) -> Optional[str]:
    """ToolPrimitive::validate (geometry/tool.rs:360): None, or the first failed check."""
    return TOOL_ERRORS[int(load_library().ix_tool_validate(C.byref(tool)))]


@dataclass
class MetricsLighting:
    """The environment the metrics score against (EnvironmentSource::Studio): a
    LightingPreset index, the rig's light yaw / pitch and the head-shadow size in
    degrees."""

    preset: int = PRESET_RING_LIGHTS
    light_yaw: float = 0.0
    light_pitch: float = 0.0
    head_shadow_deg: float = 16.0

    def to_abi(self) -> abi.MetricsLighting:
        return abi.MetricsLighting(int(self.preset), float(self.light_yaw), float(self.light_pitch),
                                   float(self.head_shadow_deg))


@dataclass
class AxisProfile:
    """AxisProfile (color/metrics/sweep.rs:20): the three 181-point curves of one axis,
    indexed by tilt away from table-up + 90 degrees (TILT_ANGLES_DEG)."""

    brilliance: np.ndarray
    extinction: np.ndarray
    windowing: np.ndarray


@dataclass
class GpuBatchItem:
    """One stone of a batch (gpu_backend/mod.rs:246): its scene, absolute sample range and
    an f64 accumulator the batch adds into."""

    scene: FrameScene
    sample_offset: int
    spp: int
    accum: np.ndarray


class GpuBackend:
    """The CUDA backend.  Thread-safe: calls from several threads are served in FIFO order
    by the library's turnstile."""

    def __init__(self, handle: Optional[int]) -> None:
        self._h = handle
        self._lib = load_library() if handle else None

    @classmethod
    def acquire(cls, device: int = 0, precision: int = abi.PRECISION_FAST,
                pipeline: GpuPipelineKind = GpuPipelineKind.MEGAKERNEL,
                threads_per_block: int = 0, chunk_paths: int = 0,
                kernel_variant: int = 0) -> "GpuBackend":
        lib = load_library()
        opts = abi.BackendOptions(device, int(pipeline), precision, threads_per_block, chunk_paths,
                                  kernel_variant)
        h = lib.ix_backend_create(C.byref(opts))
        return cls(h if h else None)

    @classmethod
    def disabled(cls) -> "GpuBackend":
        return cls(None)

    def __del__(self) -> None:
        self.close()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ix_backend_destroy(self._h)
            self._h = None

    @property
    def available(self) -> bool:
        return self._h is not None

    def adapter_label(self) -> Optional[str]:
        if not self._h:
            return None
        buf = C.create_string_buffer(256)
        self._lib.ix_backend_label(self._h, buf, 256)
        return buf.value.decode()

    def set_pipeline_kind(self, kind: GpuPipelineKind) -> None:
        if self._h:
            self._lib.ix_set_pipeline_kind(self._h, int(kind))

    def set_precision(self, precision: int) -> None:
        if self._h:
            self._lib.ix_set_precision(self._h, precision)

    def set_work_limits(self, limits: GpuWorkLimits) -> None:
        if self._h:
            wl = abi.WorkLimits(limits.max_pixels, limits.max_paths_per_call, limits.max_spp)
            self._lib.ix_set_work_limits(self._h, C.byref(wl))

    def is_lost(self) -> bool:
        return bool(self._lib.ix_is_lost(self._h)) if self._h else False

    def try_recover(self) -> bool:
        return bool(self._lib.ix_try_recover(self._h)) if self._h else True

    def last_lost_reason(self) -> Optional[str]:
        if not self._h:
            return None
        buf = C.create_string_buffer(512)
        n = self._lib.ix_last_error(self._h, buf, 512)
        return buf.value.decode() if n > 0 else None

    def last_timing(self) -> abi.TimingInfo:
        t = abi.TimingInfo()
        if self._h:
            self._lib.ix_last_timing(self._h, C.byref(t))
        return t

    def probe_fp32_peak(self) -> float:
        """Measured FP32 FMA-pipe FLOP/s of this device (FMA counted as 2)."""
        v = C.c_double(0.0)
        if not self._h or self._lib.ix_probe_fp32_peak(self._h, C.byref(v)) != 0:
            return 0.0
        return float(v.value)

    def last_dropped(self) -> int:
        return int(self._lib.ix_last_dropped(self._h)) if self._h else 0

    @staticmethod
    def _check_accum(scene: FrameScene, accum: np.ndarray) -> None:
        # GpuBackend panics on a mis-sized accumulator (gpu_backend/mod.rs:122-130).
        if accum.size != scene.width * scene.height * 3 or not accum.flags.c_contiguous:
            raise ValueError("accum must be a contiguous width*height*3 array")

    def try_accumulate_cancellable(self, scene: FrameScene, sample_offset: int, spp: int,
                                   accum: np.ndarray, cancel: Optional[CancelFlag] = None,
                                   tools: Sequence[abi.Tool] = ()) -> GpuAccumulate:
        """try_accumulate_geom_cancellable (backend.rs:272).  ``accum`` is float32 or
        float64 and is added into only on DONE; ``tools`` are the stone's concave tools
        (tool k is facet n_planes + k; when empty, the scene's own ``tools`` apply)."""
        self._check_accum(scene, accum)
        if not self._h:
            return GpuAccumulate.DECLINED
        sc = scene.to_abi()
        cp = cancel.pointer() if cancel is not None else None
        tarr = (abi.Tool * len(tools))(*tools) if tools else None
        if accum.dtype == np.float32:
            rc = self._lib.ix_accumulate(self._h, C.byref(sc), tarr, len(tools), sample_offset, spp,
                                         accum.ctypes.data_as(C.POINTER(C.c_float)), cp)
        elif accum.dtype == np.float64:
            rc = self._lib.ix_accumulate_f64(self._h, C.byref(sc), tarr, len(tools), sample_offset, spp,
                                             accum.ctypes.data_as(C.POINTER(C.c_double)), cp)
        else:
            raise TypeError("accum must be float32 or float64")
        return GpuAccumulate(rc)

    def try_accumulate_attributed(self, scene: FrameScene, lighting: "MetricsLighting", sample_offset: int,
                                  spp: int, accum: np.ndarray, attribution,
                                  cancel: Optional[CancelFlag] = None) -> GpuAccumulate:
        """try_accumulate_cancellable with spectral attribution: ``accum`` (float64) gets
        the same sums as the plain call and ``attribution`` (an
        ``attribution.AttributionMap`` of the frame's size) each sample's class and
        luminance (trace_spectral_ray_attributed_soa_geom + classify_path +
        AttributionPixel::add).  ``lighting`` is the preset / light pose / head shadow the
        scene's environment was built from.  Both are added into only on DONE."""
        self._check_accum(scene, accum)
        if accum.dtype != np.float64:
            raise TypeError("accum must be float64")
        if not self._h:
            return GpuAccumulate.DECLINED
        pixels = attribution.pixels if attribution is not None else None
        if pixels is not None and (pixels.dtype != abi.attribution_dtype() or not pixels.flags.c_contiguous):
            raise TypeError("attribution pixels must be a contiguous ix_attribution_pixel array")
        if pixels is not None and pixels.size and pixels.size != scene.width * scene.height:
            raise ValueError("attribution map must have width * height pixels")
        sc = scene.to_abi()
        cp = cancel.pointer() if cancel is not None else None
        ptr = C.c_void_p(pixels.ctypes.data) if pixels is not None and pixels.size else None
        rc = self._lib.ix_accumulate_attributed(self._h, C.byref(sc), C.byref(lighting.to_abi()), sample_offset,
                                                spp, accum.ctypes.data_as(C.POINTER(C.c_double)), ptr, cp)
        return GpuAccumulate(rc)

    def try_accumulate(self, scene: FrameScene, sample_offset: int, spp: int,
                       accum: np.ndarray) -> bool:
        """try_accumulate (backend.rs:182): True when every sample was added."""
        return self.try_accumulate_cancellable(scene, sample_offset, spp, accum) == GpuAccumulate.DONE

    def try_accumulate_batch_cancellable(self, items: Sequence[GpuBatchItem],
                                         cancel: Optional[CancelFlag] = None,
                                         on_done: Optional[Callable[[int, GpuAccumulate], None]] = None
                                         ) -> GpuAccumulate:
        """try_accumulate_batch_cancellable (backend.rs:451): each item's outcome is
        reported through ``on_done(index, outcome)`` by the library, once per item, as soon
        as that item is final."""
        if not self._h:
            for i in range(len(items)):
                if on_done:
                    on_done(i, GpuAccumulate.DECLINED)
            return GpuAccumulate.DECLINED
        arr = (abi.BatchItem * len(items))()
        scenes = []
        for i, it in enumerate(items):
            if it.accum.dtype != np.float64:
                raise TypeError("batch accumulators are float64")
            self._check_accum(it.scene, it.accum)
            sc = it.scene.to_abi()
            scenes.append(sc)
            arr[i].scene = C.pointer(sc)
            arr[i].sample_offset = it.sample_offset
            arr[i].spp = it.spp
            arr[i].accum_xyz = it.accum.ctypes.data_as(C.POINTER(C.c_double))
            arr[i].status = abi.IX_DECLINED
        cp = cancel.pointer() if cancel is not None else None
        # A NULL callback is a null function pointer of the callback's type.
        cb = (abi.BATCH_DONE_FN(lambda _u, i, st: on_done(int(i), GpuAccumulate(st))) if on_done
              else C.cast(None, abi.BATCH_DONE_FN))
        rc = self._lib.ix_accumulate_batch(self._h, arr, len(items), cp, cb, None)
        return GpuAccumulate(rc)

    def accumulate_device(self, scene_abi: abi.Scene, sample_offset: int, spp: int,
                          d_accum_ptr: int, accumulate: bool = True,
                          stream_ptr: Optional[int] = None) -> GpuAccumulate:
        """Device-resident form: ``scene_abi.planes``, its finishes and tools (if any) and
        ``d_accum_ptr`` are device pointers (a host array declines); the launch is
        enqueued on ``stream_ptr`` and not synchronised."""
        if not self._h:
            return GpuAccumulate.DECLINED
        rc = self._lib.ix_accumulate_device(self._h, C.byref(scene_abi), sample_offset, spp,
                                            C.c_void_p(d_accum_ptr), 1 if accumulate else 0,
                                            C.c_void_p(stream_ptr) if stream_ptr else None)
        return GpuAccumulate(rc)

    def evaluate_gem_optical_metrics(self, planes: np.ndarray, material: abi.Material, cam_yaw: float,
                                     cam_pitch: float, lighting: "MetricsLighting") -> Optional[np.ndarray]:
        """evaluate_gem_optical_metrics (color/metrics/evaluate.rs:158): [brilliance %,
        fire index, scintillation %, windowing %, extinction %] as float32, or None when
        the call is declined."""
        if not self._h:
            return None
        p = np.ascontiguousarray(planes, np.float32)
        out = abi.GemMetrics()
        rc = self._lib.ix_evaluate_gem_optical_metrics(self._h, p.ctypes.data_as(C.POINTER(C.c_float)),
                                                       p.shape[0], C.byref(material), cam_yaw, cam_pitch,
                                                       C.byref(lighting.to_abi()), C.byref(out))
        if rc != abi.IX_DONE:
            return None
        return np.array([out.brilliance_pct, out.fire_index, out.scintillation_pct, out.windowing_pct,
                         out.extinction_pct], np.float32)

    def evaluate_angular_profile_at_azimuth(self, planes: np.ndarray, material: abi.Material, cam_yaw: float,
                                            lighting: "MetricsLighting"):
        """evaluate_angular_profile_at_azimuth (color/metrics/profile.rs:37): (brilliance,
        extinction, windowing) float32 curves over PROFILE_ANGLES_DEG, or None when
        declined."""
        if not self._h:
            return None
        p = np.ascontiguousarray(planes, np.float32)
        out = np.zeros(3 * abi.PROFILE_ANGLES, np.float32)
        rc = self._lib.ix_evaluate_angular_profile_at_azimuth(
            self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.shape[0], C.byref(material), cam_yaw,
            C.byref(lighting.to_abi()), out.ctypes.data_as(C.POINTER(C.c_float)))
        if rc != abi.IX_DONE:
            return None
        b, e, w = out.reshape(3, abi.PROFILE_ANGLES)
        return b.copy(), e.copy(), w.copy()

    def evaluate_angular_profile(self, planes: np.ndarray, material: abi.Material, lighting: "MetricsLighting"):
        """evaluate_angular_profile (profile.rs:379): the profile at azimuth 0."""
        return self.evaluate_angular_profile_at_azimuth(planes, material, 0.0, lighting)

    def evaluate_axis_profiles(self, planes: np.ndarray, material: abi.Material, azimuths_deg: Sequence[float],
                               lighting: "MetricsLighting") -> Optional[List["AxisProfile"]]:
        """evaluate_full_axis_profile_at_azimuth (profile.rs:200) for each positive azimuth
        (degrees), all poses in one launch; None when declined."""
        if not self._h:
            return None
        p = np.ascontiguousarray(planes, np.float32)
        az = np.ascontiguousarray(azimuths_deg, np.float32)
        out = np.zeros((len(az), 3, abi.AXIS_TILTS), np.float32)
        rc = self._lib.ix_evaluate_axis_profiles(
            self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.shape[0], C.byref(material),
            az.ctypes.data_as(C.POINTER(C.c_float)), len(az), C.byref(lighting.to_abi()),
            out.ctypes.data_as(C.POINTER(C.c_float)))
        if rc != abi.IX_DONE:
            return None
        return [AxisProfile(o[0].copy(), o[1].copy(), o[2].copy()) for o in out]

    def evaluate_full_axis_profile_at_azimuth(self, planes: np.ndarray, material: abi.Material,
                                              positive_azimuth_deg: float, lighting: "MetricsLighting"):
        """evaluate_full_axis_profile_at_azimuth (profile.rs:200): (brilliance, extinction,
        windowing) over TILT_ANGLES_DEG, or None when declined."""
        r = self.evaluate_axis_profiles(planes, material, [positive_azimuth_deg], lighting)
        return None if r is None else (r[0].brilliance, r[0].extinction, r[0].windowing)

    def evaluate_all_axes_profiles(self, planes: np.ndarray, material: abi.Material,
                                   lighting: "MetricsLighting") -> Optional[List["AxisProfile"]]:
        """evaluate_all_axes_profiles (sweep.rs:74): one AxisProfile per
        PROFILE_AZIMUTHS_DEG entry (724 poses, one launch)."""
        return self.evaluate_axis_profiles(planes, material, abi.PROFILE_AZIMUTHS_DEG, lighting)

    def evaluate_metrics_batch(self, stones: Sequence[tuple], poses: Sequence[tuple], lighting: "MetricsLighting",
                               want_fire_and_scintillation: bool = True) -> Optional[np.ndarray]:
        """Many poses in one launch.  ``stones``: (planes, dispersion) pairs; ``poses``:
        (stone index, cam_yaw, cam_pitch).  Returns an (n_poses, 5) float32 array in the
        GemOpticalMetrics order, or None when declined."""
        if not self._h:
            return None
        keep = [np.ascontiguousarray(p, np.float32) for p, _ in stones]
        st = (abi.MetricsStone * len(stones))()
        for i, (p, (_, disp)) in enumerate(zip(keep, stones)):
            st[i].planes = p.ctypes.data_as(C.POINTER(C.c_float))
            st[i].n_planes = p.shape[0]
            st[i].dispersion = disp
        ps = (abi.MetricsPose * len(poses))()
        for i, (s, yaw, pitch) in enumerate(poses):
            ps[i].stone, ps[i].cam_yaw, ps[i].cam_pitch = int(s), float(yaw), float(pitch)
        out = (abi.GemMetrics * len(poses))()
        rc = self._lib.ix_evaluate_gem_optical_metrics_batch(self._h, st, len(stones), C.byref(lighting.to_abi()),
                                                             ps, len(poses), 1 if want_fire_and_scintillation else 0,
                                                             out)
        if rc != abi.IX_DONE:
            return None
        return np.frombuffer(bytes(out), np.float32).reshape(len(poses), 5).copy()

    def debug_check(self, scene: FrameScene, fn: int, inputs: np.ndarray, out_words: int) -> np.ndarray:
        """Runs per-function check kernel ``fn`` over the rows of ``inputs`` (32-bit words)."""
        if not self._h:
            raise RuntimeError("no CUDA device")
        inp = np.ascontiguousarray(inputs).view(np.uint32)
        if inp.ndim == 1:
            inp = inp.reshape(-1, 1)
        n, stride = inp.shape
        out = np.zeros((n, out_words), np.uint32)
        sc = scene.to_abi()
        rc = self._lib.ix_debug_check(self._h, C.byref(sc), fn, n,
                                      inp.ctypes.data_as(C.POINTER(C.c_uint32)), stride,
                                      out.ctypes.data_as(C.POINTER(C.c_uint32)), out_words)
        if rc != 0:
            raise RuntimeError(f"check kernel failed: {self.last_lost_reason()}")
        return out


class BatchPlan:
    """Many scenes (stones x tilts) traced by one persistent launch, replayed from a CUDA
    graph: ``run()`` enqueues every job; ``sums(j)`` is job j's per-pixel f64 sums
    (``height x width x 3``) after ``download()``."""

    def __init__(self, backend: GpuBackend, jobs: Sequence[tuple]):
        """``jobs``: (FrameScene, sample_offset, spp) per job; identical scene objects are
        uploaded once."""
        if not backend.available:
            raise RuntimeError("no CUDA backend")
        self._b = backend
        self._lib = backend._lib
        uniq, index = [], {}
        job_arr = (abi.BatchJob * len(jobs))()
        for j, (fs, off, spp) in enumerate(jobs):
            if id(fs) not in index:
                index[id(fs)] = len(uniq)
                uniq.append(fs)
            job_arr[j] = abi.BatchJob(index[id(fs)], off, spp)
        scenes = (abi.Scene * len(uniq))()
        for i, fs in enumerate(uniq):
            scenes[i] = fs.to_abi()
        self.scenes = uniq
        self.jobs = list(jobs)
        self._h = self._lib.ix_batch_plan_create(backend._h, scenes, len(uniq), job_arr, len(jobs))
        if not self._h:
            raise RuntimeError(f"batch plan declined: {backend.last_lost_reason()}")
        self.paths = int(self._lib.ix_batch_plan_paths(self._h))
        self._host = None

    def run(self, stream_ptr: Optional[int] = None) -> None:
        rc = self._lib.ix_batch_plan_run(self._h, C.c_void_p(stream_ptr) if stream_ptr else None)
        if rc != abi.IX_DONE:
            raise RuntimeError(f"batch launch declined: {self._b.last_lost_reason()}")

    def autotune(self, reps: int = 2) -> int:
        v = C.c_uint32(0)
        if self._lib.ix_batch_plan_autotune(self._h, reps, C.byref(v)) != 0:
            raise RuntimeError(f"autotune failed: {self._b.last_lost_reason()}")
        return int(v.value)

    def set_variant(self, variant: int) -> bool:
        """Pins the kernel variant (budget + 3 * shape, or 12: the wavefront pipeline);
        False when it cannot run here."""
        return self._lib.ix_batch_plan_set_variant(self._h, int(variant)) == 0

    @property
    def variant(self) -> int:
        return int(self._lib.ix_batch_plan_variant(self._h))

    def device_output(self) -> int:
        return int(self._lib.ix_batch_plan_device_output(self._h))

    def download(self) -> np.ndarray:
        n = int(self._lib.ix_batch_plan_output_size(self._h))
        host = np.zeros(n, np.float64)
        if self._lib.ix_batch_plan_download(self._h, host.ctypes.data_as(C.POINTER(C.c_double))) != 0:
            raise RuntimeError(f"download failed: {self._b.last_lost_reason()}")
        self._host = host
        return host

    def sums(self, job: int) -> np.ndarray:
        if self._host is None:
            self.download()
        fs = self.jobs[job][0]
        off = int(self._lib.ix_batch_plan_job_offset(self._h, job))
        n = fs.width * fs.height * 3
        return self._host[off:off + n].reshape(fs.height, fs.width, 3)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ix_batch_plan_destroy(self._h)
            self._h = None

    def __del__(self) -> None:
        self.close()
