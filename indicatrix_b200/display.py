"""Host-side mirror of the reference's display pipeline over ``libix_cuda.so``
(``include/ix_display.h``): the guide-buffer prepass, the edge-avoiding A-Trous denoiser
and the tone-map, with the reference's names and argument meaning
(crates/indicatrix/src/renderer/guide_pass.rs, renderer/denoise/mod.rs,
renderer/tonemap.rs, renderer/frame_denoise.rs):

* ``generate_guide_buffers(backend, width, height, camera, planes, n_d=0.0)`` ->
  ``GuideBuffers`` (depth, normal, facet_id, path_sig);
* ``AtrousDenoiser(backend).denoise_into(GBuffers, AtrousParams, output)``;
* ``tonemap_to_rgba(backend, colors, scale)`` / ``tonemap_accumulation(...)``;
* ``denoise_and_tonemap_frame(backend, FirstHitSnapshot, params)``;
* ``display_frame(backend, scene, spp, accum, with_signature)`` -- this library's own
  device-resident pipeline (guides cached per pose on the device).

Every call runs on the CUDA device; a declined call (lost device, bad arguments) returns
None / False and writes nothing.  Nothing here falls back to a CPU implementation.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import abi
from .backend import FrameScene, GpuBackend, load_library

AtrousParams = abi.AtrousParams


class DisplayTiming(C.Structure):
    """ix_display_timing: device time of the last display call's stages."""

    _fields_ = [
        ("guide_ms", C.c_float),
        ("pack_ms", C.c_float),
        ("atrous_ms", C.c_float),
        ("atrous_passes", C.c_uint32),
        ("launches", C.c_uint32),
    ]


_bound = False


def _lib() -> C.CDLL:
    global _bound
    lib = load_library()
    if not _bound:
        P = C.POINTER
        f32p, i32p, u32p, u8p = P(C.c_float), P(C.c_int32), P(C.c_uint32), P(C.c_uint8)
        lib.ix_atrous_params_default.argtypes = [P(abi.AtrousParams)]
        lib.ix_display_last_timing.argtypes = [C.c_void_p, P(DisplayTiming)]
        lib.ix_generate_guide_buffers.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, P(abi.Camera), f32p,
                                                  C.c_uint32, C.c_float, f32p, f32p, i32p, u32p]
        lib.ix_atrous_denoise.argtypes = [C.c_void_p, f32p, f32p, f32p, i32p, u32p, C.c_uint32, C.c_uint32,
                                          C.c_uint32, P(abi.AtrousParams), f32p]
        lib.ix_tonemap_to_rgba.argtypes = [C.c_void_p, f32p, C.c_uint64, C.c_float, u8p]
        lib.ix_tonemap_accumulation.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, f32p,
                                                C.c_uint32, u8p]
        lib.ix_denoise_and_tonemap_frame.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, f32p, f32p,
                                                     f32p, i32p, u32p, P(abi.AtrousParams), u8p]
        lib.ix_display_frame.argtypes = [C.c_void_p, P(abi.Scene), C.c_uint32, C.c_uint32, f32p,
                                         P(abi.AtrousParams), u8p]
        lib.ix_display_frame_device.argtypes = [C.c_void_p, P(abi.Scene), C.c_uint32, C.c_uint32, C.c_void_p,
                                                P(abi.AtrousParams), C.c_void_p, C.c_void_p]
        _bound = True
    return lib


def _p(a: Optional[np.ndarray], ctype):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def _f32(a, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and out.size != int(np.prod(shape)):
        raise ValueError(f"expected {int(np.prod(shape))} floats, got {out.size}")
    return out


@dataclass
class GuideBuffers:
    """GuideBuffers (guide_pass.rs:75): row-major [height, width] (normal [h, w, 3])."""

    depth: np.ndarray
    normal: np.ndarray
    facet_id: np.ndarray
    path_sig: np.ndarray

    @classmethod
    def miss(cls, width: int, height: int) -> "GuideBuffers":
        return cls(np.full((height, width), 1.0e6, np.float32), np.zeros((height, width, 3), np.float32),
                   np.full((height, width), -1, np.int32), np.zeros((height, width), np.uint32))


def generate_guide_buffers(backend: GpuBackend, width: int, height: int, camera: abi.Camera, planes: np.ndarray,
                           n_d: float = 0.0) -> Optional[GuideBuffers]:
    """generate_guide_buffers_with_index: one un-jittered camera ray per pixel."""
    if not backend.available:
        return None
    planes = _f32(planes)
    g = GuideBuffers(np.zeros((height, width), np.float32), np.zeros((height, width, 3), np.float32),
                     np.zeros((height, width), np.int32), np.zeros((height, width), np.uint32))
    rc = _lib().ix_generate_guide_buffers(backend._h, width, height, C.byref(camera), _p(planes, C.c_float),
                                          planes.size // 4, n_d, _p(g.depth, C.c_float), _p(g.normal, C.c_float),
                                          _p(g.facet_id, C.c_int32), _p(g.path_sig, C.c_uint32))
    return g if rc == 0 else None


@dataclass
class GBuffers:
    """GBuffers (denoise/mod.rs:118): the averaged colour plus the guides."""

    color: np.ndarray
    depth: np.ndarray
    normal: np.ndarray
    facet_id: np.ndarray
    path_sig: Optional[np.ndarray]
    width: int
    height: int
    spp: int


class AtrousDenoiser:
    """AtrousDenoiser (denoise/mod.rs:226): device buffers live in the backend and are
    reused across calls, so a kept instance allocates nothing per frame."""

    def __init__(self, backend: GpuBackend) -> None:
        self.backend = backend

    def denoise(self, inputs: GBuffers, params: Optional[AtrousParams] = None) -> Optional[np.ndarray]:
        out = np.zeros((inputs.height, inputs.width, 3), np.float32)
        return out if self.denoise_into(inputs, params, out) else None

    def denoise_into(self, inputs: GBuffers, params: Optional[AtrousParams], output: np.ndarray) -> bool:
        if not self.backend.available:
            return False
        n = inputs.width * inputs.height
        params = params if params is not None else AtrousParams.default()
        color = _f32(inputs.color, (n, 3))
        if output.dtype != np.float32 or output.size != 3 * n or not output.flags.c_contiguous:
            raise ValueError("output must be a contiguous float32 buffer of width * height * 3")
        sig = None if inputs.path_sig is None else np.ascontiguousarray(inputs.path_sig, np.uint32)
        rc = _lib().ix_atrous_denoise(self.backend._h, _p(color, C.c_float), _p(_f32(inputs.depth, (n,)), C.c_float),
                                      _p(_f32(inputs.normal, (n, 3)), C.c_float),
                                      _p(np.ascontiguousarray(inputs.facet_id, np.int32), C.c_int32),
                                      _p(sig, C.c_uint32), inputs.width, inputs.height, inputs.spp,
                                      C.byref(params), _p(output, C.c_float))
        return rc == 0


def tonemap_to_rgba(backend: GpuBackend, colors: np.ndarray, scale: float = 1.0) -> Optional[np.ndarray]:
    """tonemap_to_rgba (tonemap.rs:141): RGBA8 of xyz_to_srgb_gamma(colour * scale)."""
    colors = _f32(colors)
    n = colors.size // 3
    out = np.zeros(colors.shape[:-1] + (4,), np.uint8)
    if not backend.available:
        return None
    rc = _lib().ix_tonemap_to_rgba(backend._h, _p(colors, C.c_float), n, scale, _p(out, C.c_uint8))
    return out if rc == 0 else None


def tonemap_accumulation(backend: GpuBackend, width: int, height: int, samples_per_pixel: int, accum: np.ndarray,
                         color_space: int = abi.COLOR_SPACE_SRGB) -> Optional[np.ndarray]:
    """tonemap_accumulation (tonemap.rs:213): summed XYZ -> RGBA8 in `color_space`."""
    accum = _f32(accum, (width * height, 3))
    out = np.zeros((height, width, 4), np.uint8)
    if not backend.available:
        return None
    rc = _lib().ix_tonemap_accumulation(backend._h, width, height, samples_per_pixel, _p(accum, C.c_float),
                                        color_space, _p(out, C.c_uint8))
    return out if rc == 0 else None


@dataclass
class FirstHitSnapshot:
    """FirstHitSnapshot (frame_denoise.rs:96): an empty / None path_sig means none."""

    width: int
    height: int
    current_sample_count: int
    accum_buffer: np.ndarray
    first_hit_depth: np.ndarray
    first_hit_normal: np.ndarray
    first_hit_facet_id: np.ndarray
    first_hit_path_sig: Optional[np.ndarray] = None


def denoise_and_tonemap_frame(backend: GpuBackend, frame: FirstHitSnapshot,
                              params: Optional[AtrousParams] = None) -> Optional[np.ndarray]:
    """denoise_and_tonemap_frame_with_params_into: sRGB RGBA8 [height, width, 4]."""
    if not backend.available:
        return None
    n = frame.width * frame.height
    params = params if params is not None else AtrousParams.default()
    sig = frame.first_hit_path_sig
    sig = None if sig is None or np.size(sig) == 0 else np.ascontiguousarray(sig, np.uint32)
    out = np.zeros((frame.height, frame.width, 4), np.uint8)
    rc = _lib().ix_denoise_and_tonemap_frame(
        backend._h, frame.width, frame.height, frame.current_sample_count,
        _p(_f32(frame.accum_buffer, (n, 3)), C.c_float), _p(_f32(frame.first_hit_depth, (n,)), C.c_float),
        _p(_f32(frame.first_hit_normal, (n, 3)), C.c_float),
        _p(np.ascontiguousarray(frame.first_hit_facet_id, np.int32), C.c_int32), _p(sig, C.c_uint32),
        C.byref(params), _p(out, C.c_uint8))
    return out if rc == 0 else None


def display_frame(backend: GpuBackend, scene: FrameScene, spp: int, accum: np.ndarray, with_signature: bool = False,
                  params: Optional[AtrousParams] = None, out: Optional[np.ndarray] = None) -> Optional[np.ndarray]:
    """The whole display step of one accumulated frame on the device: guides of `scene`
    (cached per pose), average, denoise, tone-map.  `accum` is the frame's XYZ sums (the
    f64 sums of try_accumulate are rounded to f32, the reference's accumulation type).
    `out` (uint8 [height, width, 4], contiguous) is written in place when given, like the
    reference's `_into` forms; else a new array is returned."""
    if not backend.available:
        return None
    params = params if params is not None else AtrousParams.default()
    accum = _f32(accum, (scene.width * scene.height, 3))
    if out is None:
        out = np.zeros((scene.height, scene.width, 4), np.uint8)
    elif out.dtype != np.uint8 or out.size != 4 * scene.width * scene.height or not out.flags.c_contiguous:
        raise ValueError("out must be a contiguous uint8 buffer of width * height * 4")
    sc = scene.to_abi()
    rc = _lib().ix_display_frame(backend._h, C.byref(sc), 1 if with_signature else 0, spp, _p(accum, C.c_float),
                                 C.byref(params), _p(out, C.c_uint8))
    return out if rc == 0 else None


def display_frame_device(backend: GpuBackend, scene_abi: abi.Scene, spp: int, d_accum_ptr: int, d_rgba_ptr: int,
                         with_signature: bool = False, params: Optional[AtrousParams] = None,
                         stream_ptr: Optional[int] = None) -> bool:
    """Device-resident form: `d_accum_ptr` (f32 XYZ sums) and `d_rgba_ptr` are device
    pointers, enqueued on `stream_ptr` and not synchronised."""
    if not backend.available:
        return False
    params = params if params is not None else AtrousParams.default()
    rc = _lib().ix_display_frame_device(backend._h, C.byref(scene_abi), 1 if with_signature else 0, spp,
                                        C.c_void_p(d_accum_ptr), C.byref(params), C.c_void_p(d_rgba_ptr),
                                        C.c_void_p(stream_ptr) if stream_ptr else None)
    return rc == 0


def last_timing(backend: GpuBackend) -> Optional[DisplayTiming]:
    t = DisplayTiming()
    if not backend.available or _lib().ix_display_last_timing(backend._h, C.byref(t)) != 0:
        return None
    return t
