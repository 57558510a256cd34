"""Facet half-space sets built from cutting angles, in FP64.

A stone is the intersection of half-spaces ``n . x + d <= 0`` (the reference's
``GpuFacetPlane`` convention, crates/indicatrix/src/geometry/plane.rs:34-41), y up, the
girdle in the y = 0 plane.  Every plane is derived in double precision from angles,
azimuths and the point it must pass through, normalised in double, and only then
rounded to the f32 ``{nx, ny, nz, d}`` rows the transport reads.

The parametric round brilliant, the random stones and the step cut are this library's
own generators: the reference's fixed builders (geometry/cuts/round_brilliant.rs:71-155,
cuts/emerald.rs:28) do not take these parameters.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np


def _plane_through(normal: Tuple[float, float, float], point: Tuple[float, float, float]):
    n = np.asarray(normal, np.float64)
    n = n / np.linalg.norm(n)
    d = -float(np.dot(n, np.asarray(point, np.float64)))
    return (n[0], n[1], n[2], d)


def _tilted(angle_deg: float, azimuth: float, crown: bool):
    a = math.radians(angle_deg)
    return (math.sin(a) * math.cos(azimuth), math.cos(a) if crown else -math.cos(a),
            math.sin(a) * math.sin(azimuth))


@dataclass
class RoundBrilliantParams:
    """A round brilliant with ``symmetry``-fold mains (8 for the standard cut)."""

    table_pct: float = 57.0
    crown_deg: float = 34.5
    pavilion_deg: float = 40.75
    girdle_pct: float = 2.0
    girdle_segments: int = 64
    symmetry: int = 8
    star_offset_deg: float = -12.0       # star angle relative to the crown mains
    upper_half_offset_deg: float = 6.5   # upper girdle halves relative to the crown mains
    lower_half_offset_deg: float = 1.75  # lower girdle halves relative to the pavilion mains
    diameter: float = 1.0


def round_brilliant(p: RoundBrilliantParams = RoundBrilliantParams()) -> np.ndarray:
    """Round brilliant: table, ``symmetry`` crown mains, stars and 2x upper halves,
    ``girdle_segments`` vertical girdle planes, ``symmetry`` pavilion mains and 2x lower
    halves (pointed culet).  With the defaults: 57 facets + 64 girdle planes = 121."""
    R = 0.5 * p.diameter
    h = 0.5 * p.girdle_pct / 100.0 * p.diameter
    r_t = 0.5 * p.table_pct / 100.0 * p.diameter
    n = p.symmetry
    step = 2.0 * math.pi / n
    half = step / 8.0  # upper/lower halves sit 1/8 of a main sector off each main
    tc = math.radians(p.crown_deg)
    y_table = h + (R - r_t) * math.tan(tc)
    planes: List[Tuple[float, float, float, float]] = []
    planes.append((0.0, 1.0, 0.0, -y_table))
    # Stars: their top edges are the table's edges between adjacent main tips.
    star_deg = p.crown_deg + p.star_offset_deg
    edge_r = r_t * math.cos(step / 2.0)
    for m in range(n):
        phi = (m + 0.5) * step
        planes.append(_plane_through(_tilted(star_deg, phi, True),
                                     (edge_r * math.cos(phi), y_table, edge_r * math.sin(phi))))
    for m in range(n):
        phi = m * step
        planes.append(_plane_through(_tilted(p.crown_deg, phi, True),
                                     (R * math.cos(phi), h, R * math.sin(phi))))
    uh_deg = p.crown_deg + p.upper_half_offset_deg
    for m in range(n):
        for s in (-1.0, 1.0):
            phi = m * step + s * half
            planes.append(_plane_through(_tilted(uh_deg, phi, True),
                                         (R * math.cos(phi), h, R * math.sin(phi))))
    for i in range(p.girdle_segments):
        phi = 2.0 * math.pi * i / p.girdle_segments
        planes.append((math.cos(phi), 0.0, math.sin(phi), -R))
    for m in range(n):
        phi = m * step
        planes.append(_plane_through(_tilted(p.pavilion_deg, phi, False),
                                     (R * math.cos(phi), -h, R * math.sin(phi))))
    lh_deg = p.pavilion_deg + p.lower_half_offset_deg
    for m in range(n):
        for s in (-1.0, 1.0):
            phi = m * step + s * half
            planes.append(_plane_through(_tilted(lh_deg, phi, False),
                                         (R * math.cos(phi), -h, R * math.sin(phi))))
    return np.asarray(planes, np.float64)


def step_cut(length: float = 1.0, width: float = 0.7, corner_frac: float = 0.18,
             crown_deg=(50.0, 40.0, 30.0), pavilion_deg=(60.0, 50.0, 40.0),
             table_pct: float = 60.0, girdle_pct: float = 1.5) -> np.ndarray:
    """Octagonal step (emerald) cut: table, three crown tiers and three pavilion tiers of
    eight facets each (four sides and four cut corners) over a knife-edge girdle --
    1 + 24 + 24 = 49 facets.  Tier k's planes pass through the outline scaled by the
    tier's start fraction, at that tier's angle."""
    a, b = 0.5 * length, 0.5 * width
    c = corner_frac * min(a, b) * 2.0
    # Outline directions: +x, corner, +z, corner, -x, corner, -z, corner.
    outline = []
    for k in range(8):
        if k % 2 == 0:
            phi = k * math.pi / 4.0
            dist = a if k % 4 == 0 else b
        else:
            phi = k * math.pi / 4.0
            # corner chamfer: distance along the diagonal direction
            dist = (a + b - c) / math.sqrt(2.0)
        outline.append((phi, dist))
    h = 0.5 * girdle_pct / 100.0 * length
    planes = []
    tiers = len(crown_deg)
    # Crown tiers: tier t starts at scale s_t of the outline and height y_t.
    t_frac = table_pct / 100.0
    scales = [1.0 - (1.0 - t_frac) * i / tiers for i in range(tiers + 1)]
    y = h
    ys = [y]
    for t in range(tiers):
        # rise of tier t over its horizontal run at the narrowest outline distance
        run = (scales[t] - scales[t + 1]) * min(a, b)
        y += run * math.tan(math.radians(crown_deg[t]))
        ys.append(y)
    planes.append((0.0, 1.0, 0.0, -ys[-1]))
    for t in range(tiers):
        for phi, dist in outline:
            d_t = dist * scales[t]
            planes.append(_plane_through(_tilted(crown_deg[t], phi, True),
                                         (d_t * math.cos(phi), ys[t], d_t * math.sin(phi))))
    p_scales = [1.0 - i / (tiers + 0.5) for i in range(tiers)]
    y = -h
    y_p = [y]
    for t in range(tiers - 1):
        run = (p_scales[t] - p_scales[t + 1]) * min(a, b)
        y -= run * math.tan(math.radians(pavilion_deg[t]))
        y_p.append(y)
    for t in range(tiers):
        for phi, dist in outline:
            d_t = dist * p_scales[t]
            planes.append(_plane_through(_tilted(pavilion_deg[t], phi, False),
                                         (d_t * math.cos(phi), y_p[t], d_t * math.sin(phi))))
    return np.asarray(planes, np.float64)


def random_stone(rng: np.random.Generator) -> Tuple[np.ndarray, dict]:
    """One seeded random convex round stone with 33-121 facets: crown 25-45 deg,
    pavilion 37-45 deg, table 45-70 %, 4- to 8-fold mains and a girdle of enough
    segments to land in the facet range."""
    symmetry = int(rng.integers(4, 9))
    base = 1 + 7 * symmetry
    lo = max(8, 33 - base)
    hi = 121 - base
    girdle = int(rng.integers(lo, hi + 1))
    params = RoundBrilliantParams(
        table_pct=float(rng.uniform(45.0, 70.0)),
        crown_deg=float(rng.uniform(25.0, 45.0)),
        pavilion_deg=float(rng.uniform(37.0, 45.0)),
        girdle_pct=float(rng.uniform(1.0, 4.0)),
        girdle_segments=girdle,
        symmetry=symmetry,
    )
    planes = round_brilliant(params)
    return planes, {"facets": planes.shape[0], **params.__dict__}


def to_f32(planes: np.ndarray) -> np.ndarray:
    """Round the FP64 half-spaces to the f32 rows the transport reads (normal
    renormalised in f64 before rounding)."""
    p = np.asarray(planes, np.float64).copy()
    nrm = np.linalg.norm(p[:, :3], axis=1, keepdims=True)
    p[:, :3] /= nrm
    p[:, 3] /= nrm[:, 0]
    return np.ascontiguousarray(p.astype(np.float32))


def face_planes(planes: np.ndarray, tol: float = 1e-9) -> np.ndarray:
    """Boolean mask of the planes that carry a 2-D face of the polytope (FP64 vertex
    enumeration over plane triples)."""
    P = np.asarray(planes, np.float64)
    n = P.shape[0]
    N, D = P[:, :3], P[:, 3]
    idx = np.array([(i, j, k) for i in range(n) for j in range(i + 1, n) for k in range(j + 1, n)])
    A = N[idx]                       # (T, 3, 3)
    bvec = -D[idx]                   # (T, 3)
    det = np.linalg.det(A)
    ok = np.abs(det) > 1e-12
    verts = np.linalg.solve(A[ok], bvec[ok][..., None])[..., 0]
    inside = np.all(verts @ N.T + D[None, :] <= tol, axis=1)
    verts = verts[inside]
    if verts.shape[0] == 0:
        return np.zeros(n, bool)
    on = np.abs(verts @ N.T + D[None, :]) <= 1e-7
    mask = np.zeros(n, bool)
    for i in range(n):
        vi = verts[on[:, i]]
        if vi.shape[0] < 3:
            continue
        vi = np.unique(np.round(vi, 9), axis=0)
        if vi.shape[0] < 3:
            continue
        c = vi - vi[0]
        if np.linalg.matrix_rank(c, tol=1e-9) >= 2:
            mask[i] = True
    return mask


def bounding_radius(planes: np.ndarray) -> float:
    """Largest vertex distance from the origin (for camera framing)."""
    P = np.asarray(planes, np.float64)
    n = P.shape[0]
    N, D = P[:, :3], P[:, 3]
    best = 0.0
    idx = np.array([(i, j, k) for i in range(n) for j in range(i + 1, n) for k in range(j + 1, n)])
    A = N[idx]
    det = np.linalg.det(A)
    ok = np.abs(det) > 1e-12
    verts = np.linalg.solve(A[ok], (-D[idx])[ok][..., None])[..., 0]
    inside = np.all(verts @ N.T + D[None, :] <= 1e-9, axis=1)
    if np.any(inside):
        best = float(np.max(np.linalg.norm(verts[inside], axis=1)))
    return best


# ------------------------------------------------------------------------------------
# Concave tools (ToolPrimitive, crates/indicatrix/src/geometry/tool.rs:233-340): the
# constructors fill the 80-byte record in f32 as the reference does.
# ------------------------------------------------------------------------------------
TOOL_BALL, TOOL_CYLINDER, TOOL_FRUSTUM, TOOL_BICONE = 0, 1, 2, 3
SWEEP_NONE, SWEEP_ALONG_AXIS, SWEEP_ACROSS_AXIS = 0, 1, 2


def _tool(kind, centre, axis, rim, half_length, r):
    from . import abi
    t = abi.Tool()
    t.kind = kind
    t.sweep_kind = SWEEP_NONE
    t.origin[:] = [float(np.float32(x)) for x in centre] + [float(np.float32(rim))]
    t.axis[:] = [float(np.float32(x)) for x in axis] + [float(np.float32(half_length))]
    t.profile[:] = [float(np.float32(r[0])), float(np.float32(r[1])), 0.0, 0.0]
    t.sweep_dir[:] = [0.0, 0.0, 0.0, 0.0]
    return t


def tool_ball(centre, radius: float):
    """ToolPrimitive::ball: a spherical dimple."""
    return _tool(TOOL_BALL, centre, (0.0, 0.0, 1.0), radius, 0.0, (radius, radius))


def tool_cylinder(centre, axis, radius: float, half_length: float):
    """ToolPrimitive::cylinder: a capped cylinder along the unit axis."""
    return _tool(TOOL_CYLINDER, centre, axis, radius, half_length, (radius, radius))


def tool_frustum(centre, axis, r_neg: float, r_pos: float, half_length: float):
    """ToolPrimitive::frustum: radius r_neg at -half_length, r_pos at +half_length; the
    rim is their f32 mean 0.5 * (r_neg + r_pos)."""
    rim = np.float32(0.5) * (np.float32(r_neg) + np.float32(r_pos))
    return _tool(TOOL_FRUSTUM, centre, axis, rim, half_length, (r_neg, r_pos))


def tool_bicone(centre, axis, rim_radius: float, half_length: float):
    """ToolPrimitive::bicone: two cones meeting at the rim, apexes on the axis."""
    return _tool(TOOL_BICONE, centre, axis, rim_radius, half_length, (0.0, 0.0))


def with_sweep(tool, sweep: int, half_stroke: float, direction=(0.0, 0.0, 0.0)):
    """ToolPrimitive::with_sweep: the tool reciprocates +-half_stroke along its axis
    (SWEEP_ALONG_AXIS) or along `direction` across it (SWEEP_ACROSS_AXIS)."""
    tool.sweep_kind = int(sweep)
    tool.profile[2] = float(np.float32(half_stroke))
    if sweep == SWEEP_ACROSS_AXIS:
        tool.sweep_dir[:] = [float(np.float32(x)) for x in direction] + [0.0]
    else:
        tool.sweep_dir[:] = [0.0, 0.0, 0.0, 0.0]
    return tool


def any_orthonormal_vector(n):
    """glam Vec3::any_orthonormal_vector (Duff et al., JCGT 2017) in f32."""
    n = np.asarray(n, np.float32)
    sign = np.float32(-1.0) if math.copysign(1.0, float(n[2])) < 0 else np.float32(1.0)
    a = np.float32(-1.0) / (sign + n[2])
    b = (n[0] * n[1]) * a
    return np.array([b, sign + (n[1] * n[1]) * a, -n[1]], np.float32)
