"""Per-pixel spectral attribution maps (renderer/attribution_map.rs).

An ``AttributionMap`` holds one ``ix_attribution_pixel`` record per image pixel: how many
of the pixel's path-traced samples fell in each class of ``classify_path``
(color/metrics/attribution.rs:75) and the luminance each class delivered.  The CUDA
backend fills it on the device (``GpuBackend.try_accumulate_attributed``); this module is
the host side of the reference's map -- construction with its size rule, the per-sample
``add`` for samples credited on the host, totals, and the share / standard-error read-outs
the overlay draws.  Sums are float32 and formed in the reference's order.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import abi

ATTRIBUTION_CLASSES = abi.ATTRIBUTION_CLASSES
CLASS_GLARE = abi.CLASS_GLARE
CLASS_WINDOWED = abi.CLASS_WINDOWED
CLASS_RETURNED = abi.CLASS_RETURNED
CLASS_SHADOW = abi.CLASS_SHADOW
CLASS_UNLIT = abi.CLASS_UNLIT
CLASS_SIDE_EXIT = abi.CLASS_SIDE_EXIT
CLASS_NO_INTERSECTION = abi.CLASS_NO_INTERSECTION
CLASS_BUDGET = abi.CLASS_BUDGET
CLASS_KILLED = abi.CLASS_KILLED
CLASS_MISS = abi.CLASS_MISS

# MAX_DIAGNOSTIC_PIXELS (color/metrics/image_types.rs:13).
MAX_DIAGNOSTIC_PIXELS = 1_048_576

# class_index (attribution_map.rs:39-58) for the extinction reasons of
# color/metrics/image_types.rs, by name.
REASON_SLOT = {
    "ObserverShadow": CLASS_SHADOW,
    "InsufficientIllumination": CLASS_UNLIT,
    "SideExit": CLASS_SIDE_EXIT,
    "BounceBudget": CLASS_BUDGET,
    "RussianRoulette": CLASS_KILLED,
    "ScatterAbsorbed": CLASS_KILLED,
    "NoIntersection": CLASS_NO_INTERSECTION,
    "EntryBlocked": CLASS_NO_INTERSECTION,
    "Invalid": CLASS_NO_INTERSECTION,
    "None": CLASS_NO_INTERSECTION,
}

_U32_MAX = np.uint32(0xFFFFFFFF)


def _sat_inc(v) -> np.uint32:
    v = np.uint32(v)
    return v if v == _U32_MAX else np.uint32(v + np.uint32(1))


class AttributionMap:
    """AttributionMap (attribution_map.rs:185-245): ``pixels`` is a row-major array of
    ``abi.attribution_dtype()`` records."""

    def __init__(self, width: int, height: int) -> None:
        """AttributionMap::new: an empty 0 x 0 map stands in for an invalid size."""
        if self.checked_size(width, height):
            self.width, self.height = int(width), int(height)
        else:
            self.width = self.height = 0
        self.version = abi.ATTRIBUTION_VERSION
        self.pixels = np.zeros(self.width * self.height, abi.attribution_dtype())

    @staticmethod
    def checked_size(width: int, height: int) -> bool:
        """AttributionMap::checked's rule: 1 .. MAX_DIAGNOSTIC_PIXELS pixels."""
        count = int(width) * int(height)
        return 0 < count <= MAX_DIAGNOSTIC_PIXELS

    @classmethod
    def checked(cls, width: int, height: int) -> Optional["AttributionMap"]:
        return cls(width, height) if cls.checked_size(width, height) else None

    def add(self, pixel: int, class_code: int, y: float, scattered: bool = False,
            fluoresced: bool = False) -> None:
        """AttributionMap::add / AttributionPixel::add (attribution_map.rs:105-120,
        :227): ``class_code`` is a slot or CLASS_MISS; an index outside the map is
        ignored; a non-finite ``y`` counts as a hit of its class but is not summed."""
        if not 0 <= pixel < self.pixels.size:
            return
        p = self.pixels[pixel]
        p["samples"] = _sat_inc(p["samples"])
        if class_code == CLASS_MISS:
            return
        k = int(class_code)
        p["hits"] = _sat_inc(p["hits"])
        p["counts"][k] = _sat_inc(p["counts"][k])
        y32 = np.float32(y)
        if np.isfinite(y32):
            p["y_sum"][k] = np.float32(p["y_sum"][k] + y32)
            p["y_sq_sum"][k] = np.float32(p["y_sq_sum"][k] + np.float32(y32 * y32))
        p["scattered"] += np.uint32(bool(scattered))
        p["fluoresced"] += np.uint32(bool(fluoresced))

    def clear(self) -> None:
        """Forgets every sample, keeping the size."""
        self.pixels[...] = np.zeros((), abi.attribution_dtype())

    def totals(self) -> np.void:
        """The sum over all pixels in row-major order (AttributionPixel::merge, float32
        sums formed pixel by pixel)."""
        t = np.zeros((), abi.attribution_dtype())
        with np.errstate(over="ignore"):
            for name in ("samples", "hits", "scattered", "fluoresced"):
                t[name] = np.uint32(min(int(self.pixels[name].astype(np.uint64).sum()), 0xFFFFFFFF))
            t["counts"] = np.minimum(self.pixels["counts"].astype(np.uint64).sum(axis=0),
                                     0xFFFFFFFF).astype(np.uint32)
            ys = np.zeros(ATTRIBUTION_CLASSES, np.float32)
            yq = np.zeros(ATTRIBUTION_CLASSES, np.float32)
            for p in self.pixels:
                ys = (ys + p["y_sum"]).astype(np.float32)
                yq = (yq + p["y_sq_sum"]).astype(np.float32)
        t["y_sum"] = ys
        t["y_sq_sum"] = yq
        return t


def probability_share(p, k: int) -> np.float32:
    """The share of hits in class k (0 with no hits)."""
    hits = int(p["hits"])
    if hits == 0:
        return np.float32(0.0)
    return np.float32(np.float32(int(p["counts"][k])) / np.float32(hits))


def energy_share(p, k: int) -> np.float32:
    """The share of delivered luminance in class k (0 when nothing was delivered); the
    total is the float32 sum of the class sums in slot order."""
    total = np.float32(0.0)
    for v in p["y_sum"]:
        total = np.float32(total + v)
    if total > 0.0:
        return np.float32(p["y_sum"][k] / total)
    return np.float32(0.0)


def probability_error(p, k: int) -> np.float32:
    """The binomial standard error of the probability share of class k."""
    hits = int(p["hits"])
    if hits == 0:
        return np.float32(0.0)
    s = probability_share(p, k)
    return np.float32(np.sqrt(np.float32(np.float32(s * np.float32(1.0 - s)) / np.float32(hits))))


def energy_error(p, k: int) -> np.float32:
    """The standard error of the mean luminance credited to class k per hit (0 with fewer
    than two hits)."""
    hits = int(p["hits"])
    if hits < 2:
        return np.float32(0.0)
    n = np.float32(hits)
    mean = np.float32(p["y_sum"][k] / n)
    second = np.float32(p["y_sq_sum"][k] / n)
    # (-mean).mul_add(mean, second): one rounding.
    var = np.float32(np.float64(-mean) * np.float64(mean) + np.float64(second))
    var = np.float32(np.float32(max(var, np.float32(0.0)) * n) / np.float32(n - np.float32(1.0)))
    return np.float32(np.sqrt(np.float32(var / n)))
