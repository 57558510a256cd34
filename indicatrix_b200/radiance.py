"""Host-side mirror of the reference's radiance frame codec over ``libix_cuda.so``
(``include/ix_radiance.h``), with the names of crates/indicatrix-net/src/radiance/:

* ``shuffle_into`` / ``unshuffle_into`` (shuffle.rs) and ``is_valid_sample``;
* ``PayloadEncoder(encoding).encode(raw) -> EncodedPayload`` (payload.rs:99);
* ``PayloadDecoder().decode_and_add(encoding, raw_len, wire, width, height, acc)`` and
  ``decode_to_vec`` (payload.rs:205-262), raising ``RadianceError`` with the reference's
  variant name;
* ``encode_device`` / ``decode_and_add_device``: the same payloads from / into per-pixel
  sums in GPU memory (a CUDA lane's frame), through a backend.

``PayloadEncoding`` values: RAW, SHUFFLE_ZSTD (not supported by this build: encoders fall
back to Raw, decoders answer UnsupportedEncoding), SHUFFLE_LZ4.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .backend import GpuBackend, load_library

MAX_FRAME_LEN = 512 * 1024 * 1024
BYTES_PER_PIXEL = 12


class PayloadEncoding(enum.IntEnum):
    RAW = 0
    SHUFFLE_ZSTD = 1
    SHUFFLE_LZ4 = 2


class RadianceError(Exception):
    """RadianceError (radiance/mod.rs:68): ``code`` is the C code, ``name`` the variant."""

    NAMES = {1: "LengthMismatch", 3: "TooLarge", 4: "RawLenMismatch", 5: "UnsupportedEncoding",
             6: "DecompressFailed", 7: "ShortOutput", 8: "BufferTooSmall", 9: "FrameOutsideRange",
             10: "SampleCountOverrun", 16: "Declined"}

    def __init__(self, code: int) -> None:
        self.code = code
        self.name = self.NAMES.get(code, f"error {code}")
        super().__init__(self.name)


_bound = False


def _lib() -> C.CDLL:
    global _bound
    lib = load_library()
    if not _bound:
        P = C.POINTER
        u8p = P(C.c_uint8)
        lib.ix_payload_encoding_supported.argtypes = [C.c_uint32]
        lib.ix_payload_max_encoded_len.restype = C.c_size_t
        lib.ix_payload_max_encoded_len.argtypes = [C.c_size_t]
        lib.ix_radiance_shuffle.argtypes = [u8p, u8p, C.c_size_t]
        lib.ix_radiance_unshuffle.argtypes = [u8p, u8p, C.c_size_t]
        lib.ix_payload_encode.argtypes = [C.c_uint32, u8p, C.c_size_t, u8p, C.c_size_t, P(C.c_size_t),
                                          P(C.c_uint32)]
        lib.ix_payload_decode_and_add.argtypes = [C.c_uint32, C.c_uint32, u8p, C.c_size_t, C.c_uint32, C.c_uint32,
                                                  P(C.c_float), P(C.c_uint32)]
        lib.ix_payload_decode.argtypes = [C.c_uint32, C.c_uint32, u8p, C.c_size_t, C.c_uint32, C.c_uint32,
                                          P(C.c_float)]
        lib.ix_payload_encode_device.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, u8p,
                                                 C.c_size_t, P(C.c_size_t), P(C.c_uint32), C.c_void_p]
        lib.ix_payload_decode_and_add_device.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, u8p, C.c_size_t,
                                                         C.c_uint32, C.c_uint32, C.c_void_p, P(C.c_uint32),
                                                         C.c_void_p]
        _bound = True
    return lib


def _u8(b) -> np.ndarray:
    return np.frombuffer(bytes(b), np.uint8) if not isinstance(b, np.ndarray) else np.ascontiguousarray(b, np.uint8)


def _p8(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _check(rc: int) -> None:
    if rc != 0:
        raise RadianceError(rc)


def is_valid_sample(v) -> bool:
    """is_valid_sample (shuffle.rs:23): every component finite and >= 0."""
    v = np.asarray(v, np.float32)
    return bool(np.all(np.isfinite(v)) and np.all(v >= 0.0))


def shuffle_into(src, dst: np.ndarray) -> None:
    s = _u8(src)
    if dst.size != s.size:
        raise ValueError("shuffle output must match the input length")
    _check(_lib().ix_radiance_shuffle(_p8(s), _p8(dst), s.size))


def unshuffle_into(src, dst: np.ndarray) -> None:
    s = _u8(src)
    if dst.size != s.size:
        raise ValueError("unshuffle output must match the input length")
    _check(_lib().ix_radiance_unshuffle(_p8(s), _p8(dst), s.size))


def encoding_supported(encoding: int) -> bool:
    return bool(_lib().ix_payload_encoding_supported(int(encoding)))


@dataclass
class EncodedPayload:
    encoding: PayloadEncoding
    raw_len: int
    bytes: bytes


class PayloadEncoder:
    """PayloadEncoder (payload.rs:57): an unsupported encoding becomes Raw."""

    def __init__(self, encoding: PayloadEncoding) -> None:
        self.encoding = PayloadEncoding(encoding) if encoding_supported(encoding) else PayloadEncoding.RAW

    def encode(self, raw) -> EncodedPayload:
        r = _u8(raw)
        cap = int(_lib().ix_payload_max_encoded_len(r.size))
        wire = np.zeros(max(cap, 1), np.uint8)
        n, used = C.c_size_t(0), C.c_uint32(0)
        _check(_lib().ix_payload_encode(int(self.encoding), _p8(r), r.size, _p8(wire), wire.size, C.byref(n),
                                        C.byref(used)))
        return EncodedPayload(PayloadEncoding(used.value), r.size, wire[: n.value].tobytes())


class PayloadDecoder:
    """PayloadDecoder (payload.rs:180): bounded decoding into the caller's sums."""

    def decode_and_add(self, encoding: int, raw_len: int, wire, width: int, height: int, acc: np.ndarray) -> int:
        if acc.dtype != np.float32 or not acc.flags.c_contiguous or acc.size != 3 * width * height:
            raise RadianceError(1)
        w = _u8(wire)
        dropped = C.c_uint32(0)
        _check(_lib().ix_payload_decode_and_add(int(encoding), raw_len, _p8(w), w.size, width, height,
                                                acc.ctypes.data_as(C.POINTER(C.c_float)), C.byref(dropped)))
        return dropped.value

    def decode_to_vec(self, encoding: int, raw_len: int, wire, width: int, height: int) -> np.ndarray:
        w = _u8(wire)
        out = np.zeros((width * height, 3), np.float32)
        _check(_lib().ix_payload_decode(int(encoding), raw_len, _p8(w), w.size, width, height,
                                        out.ctypes.data_as(C.POINTER(C.c_float))))
        return out


def encode_device(backend: GpuBackend, encoding: int, d_sums_ptr: int, width: int, height: int,
                  stream_ptr: Optional[int] = None) -> EncodedPayload:
    """The payload of per-pixel f64 sums held on the device (`d_sums_ptr`)."""
    raw_len = width * height * BYTES_PER_PIXEL
    wire = np.zeros(max(int(_lib().ix_payload_max_encoded_len(raw_len)), 1), np.uint8)
    n, used = C.c_size_t(0), C.c_uint32(0)
    _check(_lib().ix_payload_encode_device(backend._h, int(encoding), C.c_void_p(d_sums_ptr), width, height,
                                           _p8(wire), wire.size, C.byref(n), C.byref(used),
                                           C.c_void_p(stream_ptr) if stream_ptr else None))
    return EncodedPayload(PayloadEncoding(used.value), raw_len, wire[: n.value].tobytes())


def decode_and_add_device(backend: GpuBackend, encoding: int, raw_len: int, wire, width: int, height: int,
                          d_acc_ptr: int, stream_ptr: Optional[int] = None) -> int:
    """decode_and_add into f32 sums held on the device (`d_acc_ptr`); returns the dropped
    pixel count."""
    w = _u8(wire)
    dropped = C.c_uint32(0)
    _check(_lib().ix_payload_decode_and_add_device(backend._h, int(encoding), raw_len, _p8(w), w.size, width, height,
                                                   C.c_void_p(d_acc_ptr), C.byref(dropped),
                                                   C.c_void_p(stream_ptr) if stream_ptr else None))
    return dropped.value
