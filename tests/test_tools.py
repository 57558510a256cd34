"""Concave tools in the CPU oracle and the host code, against the reference's own tests.

The reference holds no golden bits for a carved stone that travel off its GPU harness;
its tool and carve tests (crates/indicatrix/src/geometry/tool/tests.rs,
optics/raytracer/intersect_stone.rs tests) are restated here against the oracle's
functions with the reference's inputs and tolerances: validation of every field, tool
intervals that agree with point classification on seeded rays for every kind and sweep,
the grazing restart, the groove normal, the rim-wedge entry, bit identity without tools.
The transport on a carved stone then keeps the white furnace.
"""
import ctypes as C
import math

import numpy as np
import pytest

from indicatrix_b200 import abi, geometry, materials
from indicatrix_b200.geometry import (SWEEP_ACROSS_AXIS, SWEEP_ALONG_AXIS, SWEEP_NONE, TOOL_BALL, TOOL_BICONE,
                                      TOOL_CYLINDER, TOOL_FRUSTUM)


@pytest.fixture(scope="module")
def oracle():
    from oracle import ix_oracle
    return ix_oracle


def _p(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))


def unit(v):
    v = np.asarray(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


def unit_cube_planes():
    """intersect_stone.rs tests' unit cube: +-X, +-Y, +-Z at distance 0.5."""
    return np.array([[1, 0, 0, -0.5], [-1, 0, 0, -0.5], [0, 1, 0, -0.5], [0, -1, 0, -0.5],
                     [0, 0, 1, -0.5], [0, 0, -1, -0.5]], np.float32)


def tools_array(tools):
    arr = (abi.Tool * max(len(tools), 1))(*tools)
    return arr, C.cast(arr, C.POINTER(abi.Tool))


def carved_hit(oracle, planes, tools, origin, direction):
    """ixo_intersect_stone: (t, normal, facet, entering) or None."""
    arr, ptr = tools_array(tools)
    t = np.zeros(1, np.float32)
    n = np.zeros(3, np.float32)
    facet, entering = C.c_int32(), C.c_int32()
    pl = np.ascontiguousarray(planes, np.float32)
    ok = oracle.lib().ixo_intersect_stone(_p(pl), pl.shape[0], ptr, len(tools), _p(origin), _p(direction),
                                          _p(t), _p(n), C.byref(facet), C.byref(entering))
    if not ok:
        return None
    return float(t[0]), n.copy(), facet.value, entering.value


def base_tool(kind):
    """tool/tests.rs:34."""
    centre = (0.1, -0.2, 0.15)
    axis = unit([0.3, 0.5, 0.8])
    if kind == TOOL_BALL:
        return geometry.tool_ball(centre, 0.4)
    if kind == TOOL_CYLINDER:
        return geometry.tool_cylinder(centre, axis, 0.3, 0.5)
    if kind == TOOL_FRUSTUM:
        return geometry.tool_frustum(centre, axis, 0.2, 0.45, 0.5)
    return geometry.tool_bicone(centre, axis, 0.45, 0.5)


def with_sweep_kind(t, sweep):
    """tool/tests.rs:45: stroke 0.3, across-axis direction any_orthonormal_vector(axis)."""
    axis = np.array(t.axis[:3], np.float32)
    return geometry.with_sweep(t, sweep, 0.3, geometry.any_orthonormal_vector(axis))


def test_tool_record_is_80_bytes():
    """tool/tests.rs:52."""
    assert C.sizeof(abi.Tool) == 80


def test_validate_rejects_each_bad_field():
    """tool/tests.rs:75: every constructor validates (with each sweep); each broken field
    is rejected with its own error."""
    from indicatrix_b200.backend import tool_validate
    for kind in (TOOL_BALL, TOOL_CYLINDER, TOOL_FRUSTUM, TOOL_BICONE):
        good = base_tool(kind)
        assert tool_validate(good) is None
        for sweep in (SWEEP_NONE, SWEEP_ALONG_AXIS, SWEEP_ACROSS_AXIS):
            assert tool_validate(with_sweep_kind(base_tool(kind), sweep)) is None

    def broken(fn):
        t = base_tool(TOOL_CYLINDER)
        fn(t)
        return tool_validate(t)

    assert broken(lambda t: t.origin.__setitem__(0, float("nan"))) == "NonFinite"
    assert broken(lambda t: t.sweep_dir.__setitem__(1, float("inf"))) == "NonFinite"
    assert broken(lambda t: t.origin.__setitem__(3, -0.1)) == "NonPositiveRadius"
    assert broken(lambda t: (t.origin.__setitem__(3, 0.0), t.profile.__setitem__(0, 0.0),
                             t.profile.__setitem__(1, 0.0))) == "NonPositiveRadius"
    assert broken(lambda t: t.axis.__setitem__(3, 0.0)) == "NonPositiveRadius"
    assert broken(lambda t: t.profile.__setitem__(2, -0.1)) == "NonPositiveRadius"
    ball = base_tool(TOOL_BALL)
    ball.axis[3] = 0.2
    assert tool_validate(ball) == "NonPositiveRadius"
    assert broken(lambda t: t.axis.__setitem__(0, 0.9)) == "AxisNotUnit"
    across = with_sweep_kind(base_tool(TOOL_CYLINDER), SWEEP_ACROSS_AXIS)
    across.sweep_dir[:3] = list(unit([0.3, 0.5, 0.8]))
    assert tool_validate(across) == "AxisNotUnit"
    assert broken(lambda t: setattr(t, "kind", 7)) == "UnknownKind"
    assert broken(lambda t: setattr(t, "sweep_kind", 5)) == "UnknownSweep"
    assert broken(lambda t: t.pad.__setitem__(1, 3)) == "PaddingNotZero"
    assert broken(lambda t: t.profile.__setitem__(3, 1.0)) == "PaddingNotZero"
    assert broken(lambda t: t.sweep_dir.__setitem__(3, 1.0)) == "PaddingNotZero"


@pytest.mark.parametrize("kind", [TOOL_BALL, TOOL_CYLINDER, TOOL_FRUSTUM, TOOL_BICONE])
@pytest.mark.parametrize("sweep", [SWEEP_NONE, SWEEP_ALONG_AXIS, SWEEP_ACROSS_AXIS])
def test_tool_interval_agrees_with_point_classification(oracle, kind, sweep):
    """tool/tests.rs:131: on seeded rays through the tool, t lies in the ray interval
    exactly where the point is inside the tool, away from the boundary (gap < 1e-4 scale
    skipped); more than 500 of the rays hit (2000 rays here, 10000 there)."""
    lib = oracle.lib()
    tool = with_sweep_kind(base_tool(kind), sweep)
    centre = np.array(tool.origin[:3], np.float32)
    scale = max(tool.origin[3], tool.profile[0], tool.profile[1])
    rng = np.random.default_rng(0x9E3779B9 % (2 ** 32) + kind * 3 + sweep)
    hit_rays = 0
    out = np.zeros(2, np.float32)
    for _ in range(2000):
        frm = centre + unit(rng.normal(size=3)) * np.float32(3.0)
        aim = centre + unit(rng.normal(size=3)) * np.float32(0.9 * abs(rng.uniform(-1, 1)))
        d = unit(aim - frm)
        got = lib.ixo_tool_ray_interval(C.byref(tool), _p(frm), _p(d), _p(out))
        hit_rays += int(bool(got))
        for i in range(64):
            t = np.float32(1.0 + 4.0 * (i + 0.5) / 64.0)
            p = (frm + d * t).astype(np.float32)
            if lib.ixo_tool_boundary_gap(C.byref(tool), _p(p)) < 1e-4 * scale:
                continue
            inside_interval = bool(got) and out[0] <= t <= out[1]
            assert inside_interval == bool(lib.ixo_tool_contains(C.byref(tool), _p(p))), (kind, sweep, t, out)
    assert hit_rays > 500


def test_no_tools_is_bit_identical_to_the_polyhedron(oracle):
    """intersect_stone.rs:308: without tools the stone intersection is the slab's."""
    lib = oracle.lib()
    rng = np.random.default_rng(0xC0FFEE11)
    for planes in (unit_cube_planes(), np.ascontiguousarray(oracle.standard_round_brilliant())):
        for i in range(600):
            radius = 3.0 if i % 2 == 0 else 0.2
            o = unit(rng.normal(size=3)) * np.float32(radius)
            d = unit(rng.normal(size=3))
            t = np.zeros(1, np.float32)
            f = C.c_int32()
            ok = lib.ixo_intersect(_p(planes), planes.shape[0], _p(o), _p(d), _p(t), C.byref(f))
            got = carved_hit(oracle, planes, [], o, d)
            assert bool(ok) == (got is not None)
            if ok:
                assert np.float32(got[0]).tobytes() == t.tobytes() and got[2] == f.value and got[3] == -1


def test_grazing_restart_from_a_small_cylinder_does_not_self_intersect(oracle):
    """intersect_stone.rs:345: a ray restarted on a radius-0.05 cylinder cut through the
    unit cube, heading outward (grazing included), leaves through the cube."""
    planes = unit_cube_planes()
    tools = [geometry.tool_cylinder((0, 0, 0), (0, 0, 1), 0.05, 2.0)]
    rng = np.random.default_rng(0x12345678)
    n = 0
    while n < 2000:
        phi = rng.uniform(0, 2 * math.pi)
        radial = np.array([math.cos(phi), math.sin(phi), 0.0], np.float32)
        o = (radial * np.float32(0.05) + np.array([0, 0, 1], np.float32) * np.float32(0.3 * rng.uniform(-1, 1)))
        tangent = np.array([-radial[1], radial[0], 0.0], np.float32)
        d = unit(radial * (0.05 + abs(rng.uniform(-1, 1))) + tangent * rng.uniform(-1, 1)
                 + np.array([0, 0, 1.0]) * rng.uniform(-1, 1))
        if float(np.dot(d, radial)) <= 0.0:
            continue
        n += 1
        hit = carved_hit(oracle, planes, tools, o.astype(np.float32), d)
        assert hit is not None and hit[2] < planes.shape[0], hit


def test_stone_hit_normal_on_a_tool_points_into_the_cavity(oracle):
    """intersect_stone.rs:377: a groove (radius 0.2 along Z, centred on the cube's top
    face) met from above: tool facet id 6, normal facing the ray, the floor at
    0.5 - sqrt(0.04 - x^2); beside the groove the top plane (facet 2)."""
    planes = unit_cube_planes()
    tools = [geometry.tool_cylinder((0.0, 0.5, 0.0), (0, 0, 1), 0.2, 2.0)]
    for x in (-0.15, -0.05, 0.0, 0.1, 0.18):
        o = np.array([x, 2.0, 0.1], np.float32)
        d = np.array([0, -1, 0], np.float32)
        t, n, facet, entering = carved_hit(oracle, planes, tools, o, d)
        assert facet == 6 and float(np.dot(n, d)) < 0.0
        expected_y = 0.5 - math.sqrt(0.2 * 0.2 - x * x)
        assert abs((o + d * np.float32(t))[1] - expected_y) < 1e-4
    hit = carved_hit(oracle, planes, tools, np.array([0.4, 2.0, 0.1], np.float32), np.array([0, -1, 0], np.float32))
    assert hit[2] == 2


def test_a_restart_across_a_tool_rim_wedge_reports_an_entry(oracle):
    """intersect_stone.rs:425: a ray restarted in the rim wedge of a ball on the cube's
    top face meets the ball's far side as an entry at t 0.60005; from inside the material
    it meets the ball as an exit; without tools no side is reported."""
    planes = unit_cube_planes()
    tools = [geometry.tool_ball((0.0, 0.5, 0.0), 0.3)]
    d = np.array([-1, 0, 0], np.float32)
    t, n, facet, entering = carved_hit(oracle, planes, tools, np.array([0.30005, 0.4999, 0.0], np.float32), d)
    assert facet == 6 and abs(t - 0.60005) < 1e-4 and entering == 1 and float(np.dot(n, d)) < 0.0
    t, n, facet, entering = carved_hit(oracle, planes, tools, np.array([0.4, 0.4, 0.0], np.float32), d)
    assert facet == 6 and entering == 0 and float(np.dot(n, d)) > 0.0
    assert carved_hit(oracle, planes, [], np.array([0.4, 0.4, 0.0], np.float32), d)[3] == -1


def carved_round_brilliant_tools():
    """A table dimple and a crown groove on the standard round brilliant (table at
    y = 0.32, girdle radius 1), the shape of the reference harness's concave image
    comparison."""
    return [geometry.tool_ball((0.0, 0.32, 0.0), 0.22),
            geometry.with_sweep(geometry.tool_cylinder((0.72, 0.14, 0.0), (0, 0, 1), 0.07, 0.4),
                                SWEEP_ALONG_AXIS, 0.1)]


def test_carved_stone_white_furnace(oracle):
    """A colourless, non-dispersive carved stone (n 1.5, a table dimple and a crown
    groove) in a uniform environment returns the environment's radiance within 0.025
    (white_furnace_energy_conservation.rs), and the carve changes the image."""
    from test_frosted import furnace_scene, furnace_target

    mat = materials.isotropic(materials.cauchy(1.5, 0.0, 0.0))
    sc, keep = furnace_scene(oracle, mat, finishes=False)
    tools = carved_round_brilliant_tools()
    arr, ptr = tools_array(tools)
    sc.tools, sc.n_tools = ptr, len(tools)
    _, s64, dropped = oracle.trace_frame(sc, 0, 96, threads=0)
    assert dropped == 0
    mean = s64.reshape(-1, 3).sum(axis=0) / (12 * 12 * 96)
    target = furnace_target(oracle)
    assert np.all(np.abs(mean - target) / target <= 0.025), (mean, target)
    plain, keep2 = furnace_scene(oracle, mat, finishes=False)
    _, p64, _ = oracle.trace_frame(plain, 0, 96, threads=0)
    assert not np.array_equal(s64, p64)


def test_routing_with_tools():
    """scene_routes_to_gpu_with_tools (tool_routing.rs:81): valid tools route, an invalid
    tool or more than IX_MAX_TOOLS decline; the scene's own tools count the same."""
    from indicatrix_b200 import backend as bk, workloads
    fs = workloads.round_brilliant_frame(8, 8)
    tools = carved_round_brilliant_tools()
    assert bk.scene_routes_to_gpu_with_tools(fs, tools)
    bad = geometry.tool_ball((0, 0, 0), 0.1)
    bad.pad[0] = 1
    assert not bk.scene_routes_to_gpu_with_tools(fs, tools + [bad])
    assert not bk.scene_routes_to_gpu_with_tools(fs, [geometry.tool_ball((0, 0, 0), 0.01)] * (abi.MAX_TOOLS + 1))
    fs.tools = tools
    assert bk.scene_routes_to_gpu(fs)
    fs.tools = tools + [bad]
    assert not bk.scene_routes_to_gpu(fs)
