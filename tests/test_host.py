"""Host-side checks that need no GPU: the C-ABI library loads and exports every symbol
``include/*.h`` declares, the ctypes structures match the C layout, the host scene
builders round exactly as the oracle's restatement of the reference does, the routing
predicate, the decline-without-device behaviour, and the FP64 geometry generators."""
import ctypes as C
import math
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from indicatrix_b200 import abi, geometry, materials, workloads
from indicatrix_b200.display import DisplayTiming
from indicatrix_b200.surrogate import DesignView
from indicatrix_b200.backend import (CancelFlag, FrameScene, GpuAccumulate, GpuBackend, camera_new,
                                     environment_preset, load_library, scene_routes_to_gpu,
                                     scene_routes_to_gpu_with_tools)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(ix_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = load_library()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n


def test_abi_struct_layout_matches_c():
    """Compile a tiny C program against include/ix_cuda.h and compare sizeof/offsetof."""
    checks = {
        "ix_camera": abi.Camera, "ix_dispersion": abi.Dispersion, "ix_band": abi.Band,
        "ix_absorption": abi.Absorption, "ix_material": abi.Material,
        "ix_environment": abi.Environment, "ix_scene": abi.Scene,
        "ix_backend_options": abi.BackendOptions, "ix_work_limits": abi.WorkLimits,
        "ix_batch_item": abi.BatchItem, "ix_timing": abi.TimingInfo,
        "ix_gem_metrics": abi.GemMetrics, "ix_metrics_lighting": abi.MetricsLighting,
        "ix_metrics_stone": abi.MetricsStone, "ix_metrics_pose": abi.MetricsPose,
        "ix_attribution_pixel": abi.AttributionPixel,
        "ix_atrous_params": abi.AtrousParams, "ix_display_timing": DisplayTiming,
        "ix_tool": abi.Tool, "ix_design_view": DesignView,
    }
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "ix_cuda.h"', '#include "ix_display.h"',
           '#include "ix_design.h"', "int main(void){", 'printf("ix_design %zu\\n", sizeof(ix_design));']
    for cname, py in checks.items():
        src.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            src.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.split() for line in out if line)
    assert int(got["ix_design"]) == 4 * 12  # 12 f32 parameters, passed as float rows
    for cname, py in checks.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def test_host_builders_match_oracle_bits(oracle):
    """ix_camera_new / ix_environment_preset (product host code) vs the oracle's own
    restatement of Camera::new, StudioRig::new, head_shadow_cosines and the blackbody
    white balance: identical bits."""
    for yaw, pitch, dist, fov in [(0.6, 0.45, 2.4, 42.0), (0.0, float(np.float32(math.pi / 2)), 1.6, 42.0),
                                  (0.35, 0.28, 5.0, 18.0), (2.0, -0.3, 3.0, 30.0)]:
        a, b = camera_new(yaw, pitch, dist, fov), oracle.camera_new(yaw, pitch, dist, fov)
        assert bytes(a) == bytes(b)
    for preset in range(15):
        for hs in (16.0, 20.0, 0.0, 2.0, 90.0):
            a = environment_preset(preset, 1.3, 0.85, 0.95, 0.2, 0.7, hs)
            b = oracle.environment_preset(preset, 1.3, 0.85, 0.95, 0.2, 0.7, hs)
            assert bytes(a) == bytes(b), (preset, hs)
    with pytest.raises(ValueError):
        environment_preset(15)


def test_routing_predicate():
    fs = workloads.round_brilliant_frame(8, 8)
    assert scene_routes_to_gpu(fs)
    for m in (materials.sapphire(), materials.quartz(), materials.rutile((0.6, 0.8, 0.0))):
        assert scene_routes_to_gpu(FrameScene(fs.camera, 8, 8, fs.planes, m, 32, fs.environment))
    m = materials.quartz()
    m.e_dispersion.kind = 7
    assert not scene_routes_to_gpu(FrameScene(fs.camera, 8, 8, fs.planes, m, 32, fs.environment))
    # Interior scattering (isotropic and uniaxial) and rounded facet edges route.
    for m in (materials.diamond(), materials.sapphire()):
        m = materials.with_scattering(m, 0.5, 0.3)
        assert scene_routes_to_gpu(FrameScene(fs.camera, 8, 8, fs.planes, m, 32, fs.environment))
    m = materials.diamond()
    m.edge_rounding_radius = 0.01
    assert scene_routes_to_gpu(FrameScene(fs.camera, 8, 8, fs.planes, m, 32, fs.environment))
    # Frosted facets route (apply_frosted_bounce runs on the device).
    fin = np.zeros(fs.planes.shape[0], np.uint8)
    fin[70] = 1
    assert scene_routes_to_gpu(FrameScene(fs.camera, 8, 8, fs.planes, materials.diamond(), 32,
                                          fs.environment, fin))
    huge = FrameScene(fs.camera, 65536, 65536, fs.planes, materials.diamond(), 32, fs.environment)
    assert not scene_routes_to_gpu(huge)  # 2^32 pixels: beyond 32-bit pixel indices
    assert scene_routes_to_gpu(FrameScene(fs.camera, 65535, 65537, fs.planes, materials.diamond(), 32,
                                          fs.environment))
    too_many = np.zeros((129, 4), np.float32)
    too_many[:, 1] = 1.0
    assert not scene_routes_to_gpu(FrameScene(fs.camera, 8, 8, too_many, materials.diamond(), 32,
                                              fs.environment))


def test_disabled_backend_declines_and_leaves_accum():
    b = GpuBackend.disabled()
    fs = workloads.round_brilliant_frame(4, 4)
    acc = np.full((4, 4, 3), 3.0)
    assert b.try_accumulate_cancellable(fs, 0, 4, acc) == GpuAccumulate.DECLINED
    assert not b.try_accumulate(fs, 0, 4, acc)
    assert np.all(acc == 3.0)
    assert b.adapter_label() is None and not b.is_lost() and b.try_recover()


def test_round_brilliant_generator():
    p = geometry.round_brilliant()
    assert p.shape == (121, 4)
    assert geometry.face_planes(p).all()
    f = geometry.to_f32(p)
    assert f.dtype == np.float32
    assert np.allclose(np.linalg.norm(f[:, :3], axis=1), 1.0, atol=1e-6)
    # table at 57 %: the crown mains reach the table plane at radius 0.285
    y_t = -p[0, 3]
    assert abs(y_t - (0.01 + (0.5 - 0.285) * math.tan(math.radians(34.5)))) < 1e-12
    # pavilion depth from the 40.75-degree mains (pointed culet)
    assert abs(geometry.bounding_radius(p) - 0.5) < 0.01


def test_step_cut_and_random_stones():
    e = geometry.step_cut()
    assert e.shape[0] == 49 and geometry.face_planes(e).all()
    stones = workloads.random_stones(16, seed=3)
    assert len(stones) == 16
    for i, st in enumerate(stones):
        assert 33 <= st.info["facets"] <= 121
        assert 25.0 <= st.info["crown_deg"] <= 45.0 and 37.0 <= st.info["pavilion_deg"] <= 45.0
        assert 45.0 <= st.info["table_pct"] <= 70.0
        assert st.spp in (32, 64, 128, 256)
        assert bool(st.material.abs_o.has_spline) == (i % 2 == 1)
        assert geometry.face_planes(st.planes.astype(np.float64)).all()


def test_tools_route_and_the_abi_forms_of_cancel_and_on_done():
    """The boundary's argument forms: an ix_tool is the reference's 80-byte ToolPrimitive;
    a valid tool routes and one failing ToolPrimitive::validate declines (here a ball
    record with a zero axis, tool_routing.rs:81); the cancel
    flag is one byte, as a Rust AtomicBool; a CTA size other than 0 / 64 / 128 / 256 and an
    unknown kernel variant are refused at create time (no device is needed to see that);
    on_done reports every item of a declined batch."""
    assert C.sizeof(abi.Tool) == 80
    fs = workloads.round_brilliant_frame(8, 8)
    assert scene_routes_to_gpu_with_tools(fs, [])
    ball = abi.Tool()
    ball.kind = 0
    ball.origin[:] = [0.0, 0.3, 0.0, 0.05]
    assert not scene_routes_to_gpu_with_tools(fs, [ball])
    assert scene_routes_to_gpu_with_tools(fs, [geometry.tool_ball((0.0, 0.3, 0.0), 0.05)])
    flag = CancelFlag()
    assert C.sizeof(flag._word) == 1 and not flag.is_set()
    flag.set()
    assert flag.is_set() and flag.pointer().contents.value == 1
    lib = load_library()
    for tpb, variant in ((96, 0), (512, 0), (0, 13)):
        opts = abi.BackendOptions(0, 0, 0, tpb, 0, variant)
        assert not lib.ix_backend_create(C.byref(opts))
    from indicatrix_b200.backend import GpuBatchItem

    seen = []
    items = [GpuBatchItem(fs, 0, 4, np.zeros((8, 8, 3))) for _ in range(3)]
    assert GpuBackend.disabled().try_accumulate_batch_cancellable(
        items, None, lambda i, r: seen.append((i, r))) == GpuAccumulate.DECLINED
    assert seen == [(i, GpuAccumulate.DECLINED) for i in range(3)]
