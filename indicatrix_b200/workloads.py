"""The benchmark workloads as concrete, seeded synthetic scenes.

* ``round_brilliant_frame``: a 121-plane round brilliant (table 57 %, crown 34.5 deg,
  pavilion 40.75 deg, 8 + 8 + 16 crown, 8 + 16 pavilion, 64-segment girdle 2 % thick,
  girdle diameter 1.0) in Diamond (Peter 1923 Sellmeier), face up under a D65 uniform
  hemisphere with a 20-degree head shadow, 42-degree pinhole camera, max depth 32.
* ``random_stones``: seeded random convex round stones, 33-121 facets, crown 25-45 deg,
  pavilion 37-45 deg, table 45-70 %, Cauchy or Sellmeier materials with n_D in
  [1.45, 2.60] and dispersion in [0.01, 0.07], half of them with a smooth 16-knot
  absorption spline of 0-5 /cm, each at 9 tilts 0-40 deg.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

from . import abi, backend, geometry, materials
from .backend import FrameScene, PRESET_ISO_HEMISPHERE

FACE_UP_PITCH = np.float32(math.pi / 2.0)
DEFAULT_FOV_DEG = 42.0
FACE_UP_DISTANCE = 1.6
# Model units per centimetre of a 1.0-diameter stone: a 6.5 mm girdle.
CM_PER_MODEL_UNIT = 0.65


# The host formulas that turn a pose into a camera and a lighting preset into an
# environment (Camera::new, EnvironmentSource::Studio): by default this library's
# (ix_camera_new / ix_environment_preset).  Any object with the same two functions --
# camera_new(yaw, pitch, distance, fov_deg) and environment_preset(preset, exposure,
# light_yaw, light_pitch, backdrop, surface_glare, head_shadow_deg) -- can stand in for it,
# e.g. a CPU implementation that must not load the CUDA library.
class _LibraryBuilder:
    camera_new = staticmethod(backend.camera_new)
    environment_preset = staticmethod(backend.environment_preset)


LIBRARY_BUILDER = _LibraryBuilder()


def iso_hemisphere(head_shadow_deg: float = 20.0, builder=None) -> abi.Environment:
    b = builder or LIBRARY_BUILDER
    return b.environment_preset(PRESET_ISO_HEMISPHERE, 1.0, 0.0, 0.0, 0.0, 1.0, head_shadow_deg)


def round_brilliant_frame(width: int = 256, height: int = 256, max_bounces: int = 32, builder=None) -> FrameScene:
    b = builder or LIBRARY_BUILDER
    planes = geometry.to_f32(geometry.round_brilliant())
    cam = b.camera_new(0.0, float(FACE_UP_PITCH), FACE_UP_DISTANCE, DEFAULT_FOV_DEG)
    return FrameScene(camera=cam, width=width, height=height, planes=planes,
                      material=materials.diamond(), max_bounces=max_bounces,
                      environment=iso_hemisphere(builder=b))


def carved_sun_frame(width: int = 256, height: int = 256, max_bounces: int = 32, builder=None) -> FrameScene:
    """The round brilliant with its table and girdle frosted and a spherical dimple (radius
    0.11) ground into the table, under the DaylightSun model at light yaw 0.4, pitch 0.5,
    seen from 0.6 rad above the girdle plane: every feature of the extended transport at
    once (the carved-stone intersection, frosted facets with next-event estimation toward
    the sun's disc, the extended environment lookup)."""
    b = builder or LIBRARY_BUILDER
    planes = geometry.to_f32(geometry.round_brilliant())
    ny = planes[:, 1]
    finishes = ((np.abs(ny) < 0.05) | (ny > 0.99)).astype(np.uint8)
    table_y = float(-planes[int(np.argmax(ny)), 3])
    cam = b.camera_new(0.4, 0.6, FACE_UP_DISTANCE, DEFAULT_FOV_DEG)
    fs = FrameScene(camera=cam, width=width, height=height, planes=planes, material=materials.diamond(),
                    max_bounces=max_bounces, environment=b.environment_preset(6, 1.0, 0.4, 0.5, 0.0, 1.0, 16.0),
                    facet_finishes=finishes)
    fs.tools = [geometry.tool_ball((0.0, table_y, 0.0), 0.11)]
    return fs


@dataclass
class StoneSpec:
    planes: np.ndarray
    material: abi.Material
    spp: int
    info: dict


def random_material(rng: np.random.Generator, absorbing: bool) -> abi.Material:
    """Cauchy or Sellmeier-1 with n_D ~ U(1.45, 2.60) and an Abbe-like dispersion
    n_F - n_C ~ U(0.01, 0.07); optional smooth absorption spline in 1/cm."""
    n_d = float(rng.uniform(1.45, 2.60))
    disp = float(rng.uniform(0.01, 0.07))
    lf, lc, ld = 0.4861, 0.6563, 0.5893  # um
    if rng.uniform() < 0.5:
        # Cauchy n = A + B / l^2 : n_F - n_C = B (1/lf^2 - 1/lc^2).
        b = disp / (1.0 / lf ** 2 - 1.0 / lc ** 2)
        a = n_d - b / ld ** 2
        d = materials.cauchy(a, b, 0.0)
    else:
        # Sellmeier-1 n^2 = 1 + B l^2 / (l^2 - C): solve C from the dispersion, then B.
        def n_of(B, C, l):
            return math.sqrt(1.0 + B * l * l / (l * l - C))

        def fit(C):
            B = (n_d ** 2 - 1.0) * (ld ** 2 - C) / ld ** 2
            return n_of(B, C, lf) - n_of(B, C, lc) - disp, B

        lo, hi = 1e-5, 0.12
        for _ in range(80):
            mid = 0.5 * (lo + hi)
            if fit(mid)[0] > 0:
                hi = mid
            else:
                lo = mid
        C = 0.5 * (lo + hi)
        B = fit(C)[1]
        d = abi.Dispersion()
        d.kind = abi.DISP_SELLMEIER1
        d.b[:] = [B, 0.0, 0.0]
        d.c[:] = [C, 0.0, 0.0]
    spline = None
    if absorbing:
        knots = rng.uniform(0.0, 1.0, abi.SPLINE_KNOTS)
        # smooth: average neighbours, scale to a random peak in [0, 5] /cm
        knots = np.convolve(np.pad(knots, 2, mode="edge"), np.ones(5) / 5.0, mode="valid")
        knots = knots / max(knots.max(), 1e-6) * rng.uniform(0.0, 5.0)
        spline = knots.astype(np.float32)
    return materials.isotropic(d, spline, path_scale=CM_PER_MODEL_UNIT)


def random_stones(n: int, seed: int = 20251203) -> List[StoneSpec]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        planes, info = geometry.random_stone(rng)
        mat = random_material(rng, absorbing=(i % 2 == 1))
        spp = int(rng.choice([32, 64, 128, 256]))
        out.append(StoneSpec(geometry.to_f32(planes), mat, spp, info))
    return out


def smooth_spline(rng: np.random.Generator, peak_max: float) -> np.ndarray:
    """A seeded smooth 16-knot absorption curve with a random peak in [0, peak_max]."""
    knots = rng.uniform(0.0, 1.0, abi.SPLINE_KNOTS)
    knots = np.convolve(np.pad(knots, 2, mode="edge"), np.ones(5) / 5.0, mode="valid")
    return (knots / max(knots.max(), 1e-6) * rng.uniform(0.0, peak_max)).astype(np.float32)


def stress_material(seed: int = 7, tilt_deg: float = 30.0) -> abi.Material:
    """The anisotropic stress material: corundum o-ray and e-ray Sellmeier fits
    (Malitson & Dodge 1972; n_o = 1.768, n_e = 1.760 at the D line), optic axis tilted
    `tilt_deg` from the table normal toward +x, and a pleochroic absorption tensor whose
    o-ray and e-ray coefficients are two seeded smooth 16-knot splines of 0-8 /cm."""
    rng = np.random.default_rng(seed)
    t = math.radians(tilt_deg)
    m = materials.uniaxial(
        materials.sellmeier3([1.4313493, 0.65054713, 5.3414021], [0.0726631 ** 2, 0.1193242 ** 2, 18.028251 ** 2]),
        -0.0081, (math.sin(t), math.cos(t), 0.0),
        e_dispersion=materials.sellmeier3([1.5039759, 0.55069141, 6.5927379],
                                          [0.0740288 ** 2, 0.1216529 ** 2, 20.072248 ** 2]))
    for ab in (m.abs_o, m.abs_e):
        ab.has_spline = 1
        ab.spline[:] = [float(x) for x in smooth_spline(rng, 8.0)]
    m.absorption_path_scale = CM_PER_MODEL_UNIT
    return m


def anisotropic_stress_frame(width: int = 512, height: int = 512, max_bounces: int = 64,
                             seed: int = 7, builder=None) -> FrameScene:
    """The emerald step cut (3 crown + 3 pavilion tiers, 49 facets) in the stress
    material, face up under the D65 hemisphere with the 20-degree head shadow, max depth 64."""
    b = builder or LIBRARY_BUILDER
    planes = geometry.to_f32(geometry.step_cut())
    cam = b.camera_new(0.0, float(FACE_UP_PITCH), FACE_UP_DISTANCE, DEFAULT_FOV_DEG)
    return FrameScene(camera=cam, width=width, height=height, planes=planes,
                      material=stress_material(seed), max_bounces=max_bounces,
                      environment=iso_hemisphere(builder=b))


TILTS_DEG = [0.0, 5.0, 10.0, 15.0, 20.0, 25.0, 30.0, 35.0, 40.0]


def tilted_scene(stone: StoneSpec, tilt_deg: float, width: int = 128, height: int = 128,
                 max_bounces: int = 32, builder=None) -> FrameScene:
    """The stone seen face-up with the camera tilted `tilt_deg` from the table normal."""
    b = builder or LIBRARY_BUILDER
    pitch = float(np.float32(math.pi / 2.0 - math.radians(tilt_deg)))
    cam = b.camera_new(0.0, pitch, FACE_UP_DISTANCE, DEFAULT_FOV_DEG)
    return FrameScene(camera=cam, width=width, height=height, planes=stone.planes,
                      material=stone.material, max_bounces=max_bounces,
                      environment=iso_hemisphere(builder=b))
