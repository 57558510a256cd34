"""Next-event estimation toward the DaylightSun disc at frosted facets, on a B200 against
the CPU oracle through the C ABI (nee_contribution_frosted_exterior,
scattering/frosted.rs:98; the escape's balance weight, bounce_body/miss.rs:40).

The round brilliant with a bruted girdle and a frosted table under a low sun: per path in
the exact build for isotropic, uniaxial and biaxial materials, a carved stone (whose
light samples are shadow-probed) and scattering stones (whose Henyey-Greenstein events
take no light sample under the analytic sun); paths cut at the bounce cap keep their
light samples (at one bounce a stone pixel is lit by next-event estimation alone); frame
sums through the accumulate entry; Tier 3 of the benched build.  As in test_gpu_frosted, the diffuse
lobe's and the disc draw's sin/cos round a few ULP apart between the device and the host
libm, so the per-path bars are the frosted ones.
"""
import numpy as np
import pytest

from indicatrix_b200 import materials
from indicatrix_b200.backend import BatchPlan, FrameScene, environment_preset

from test_frosted import bruted_girdle_finishes
from test_gpu_fast_parity import TIER3_H, TIER3_SPP, TIER3_W, oracle_moments, passes_z_criteria, z_components
from test_gpu_parity import trace_paths
from test_tools import carved_round_brilliant_tools

pytestmark = pytest.mark.gpu

CASES = {
    "diamond": lambda: materials.diamond(),
    "sapphire_tilted": lambda: materials.sapphire((0.0, 0.8, 0.6)),
    "tanzanite": lambda: materials.tanzanite((0.3, 0.8, 0.52)),
    "carved_diamond": lambda: materials.diamond(),
    # A Henyey-Greenstein event takes no light sample under the analytic sun
    # (scattering/hg_nee.rs:165); the frosted facets of the scattering stone still do.
    "scattering_diamond": lambda: materials.with_scattering(materials.diamond(), 0.5, 0.3),
    "scattering_sapphire": lambda: materials.with_scattering(materials.sapphire((0.0, 0.8, 0.6)), 0.5, 0.3),
}


def sun_scene(oracle, material, width=40, height=40, max_bounces=32, preset=6, tools=None):
    """A frosted table and bruted girdle, seen from 0.6 rad above the girdle plane, under
    the sun (or, preset 5, the same sky without it) at light yaw 0.4, pitch 0.5."""
    planes = np.ascontiguousarray(oracle.standard_round_brilliant())
    fin = bruted_girdle_finishes(planes.shape[0])
    fin[0] = 1
    cam = oracle.camera_new(0.4, 0.6, 2.2, 30.0)
    fs = FrameScene(cam, width, height, planes, material, max_bounces, environment_preset(preset, 1.0, 0.4, 0.5), fin)
    fs.tools = tools
    return fs


@pytest.mark.parametrize("name", list(CASES))
def test_sun_nee_paths_match_oracle(exact_backend, oracle, name):
    """Per path on identical (pixel, sample) inputs, exact build: >= 99 % within 1e-3
    relative and within 1e-2, the same bounce count on >= 98 %, the total within 1 %."""
    tools = carved_round_brilliant_tools() if name.startswith("carved") else None
    fs = sun_scene(oracle, CASES[name](), tools=tools)
    n = fs.width * fs.height
    xyz_o, bounces_o = oracle.trace_samples(fs.to_abi(), 0, n, 0, 8)
    xyz_g, bounces_g = trace_paths(exact_backend, fs, np.repeat(np.arange(n), 8), np.tile(np.arange(8), n))
    xo = xyz_o.reshape(-1, 3).astype(np.float64)
    xg = xyz_g.astype(np.float64)
    rel = np.abs(xg - xo).max(axis=1) / np.maximum(np.abs(xo).max(axis=1), 1e-3)
    stats = (np.mean(rel <= 1e-3), np.mean(rel <= 1e-2), np.mean(bounces_g == bounces_o.ravel()))
    assert stats[0] >= 0.99 and stats[1] >= 0.99 and stats[2] >= 0.98, (name, stats)
    assert abs(xg.sum() - xo.sum()) <= 1e-2 * xo.sum()


def test_capped_paths_keep_their_light_samples(exact_backend, oracle):
    """At max_bounces 1 a path that meets the stone ends at the cap without escaping: under
    the sky alone (DaylightDome) every such path is black, under the sun the frosted
    facets' light samples light some of them, on the device as in the oracle."""
    lit = {}
    for preset in (5, 6):
        fs = sun_scene(oracle, materials.diamond(), 32, 32, max_bounces=1, preset=preset)
        n = fs.width * fs.height
        xyz_o, _ = oracle.trace_samples(fs.to_abi(), 0, n, 0, 8)
        xyz_g, _ = trace_paths(exact_backend, fs, np.repeat(np.arange(n), 8), np.tile(np.arange(8), n))
        xo = xyz_o.reshape(-1, 3)
        assert np.allclose(xyz_g, xo, rtol=1e-3, atol=1e-6)
        lit[preset] = int(np.count_nonzero(xo[:, 1] > 0.0))
    assert lit[6] > lit[5] + 100, lit


def test_sun_nee_frame_sums(exact_backend, oracle):
    """ix_accumulate_f64 under the sun: the per-pixel sums agree with the oracle's."""
    fs = sun_scene(oracle, materials.diamond(), 40, 32)
    acc = np.zeros((32, 40, 3))
    assert exact_backend.try_accumulate(fs, 0, 32, acc)
    _, s64, dropped = oracle.trace_frame(fs.to_abi(), 0, 32)
    assert dropped == 0
    rel = (np.abs(acc - s64) / np.maximum(np.abs(s64).max(axis=2, keepdims=True), 1e-3)).max(axis=2)
    assert np.mean(rel <= 1e-3) >= 0.95
    assert abs(acc.sum() - s64.sum()) / s64.sum() < 1e-2


@pytest.mark.parametrize("name", ["diamond", "carved_diamond", "scattering_diamond"])
def test_sun_nee_tier3_fast_build(backend, oracle, name):
    """Tier 3 on the benched build: the batch plan's means over samples [0, 500) against
    the oracle's [500, 1000), each side's own variance."""
    W, H, N = TIER3_W, TIER3_H, TIER3_SPP
    tools = carved_round_brilliant_tools() if name.startswith("carved") else None
    fs = sun_scene(oracle, CASES[name](), W, H, tools=tools)
    plan = BatchPlan(backend, [(fs, 0, N)])
    plan.run()
    mg = plan.sums(0).reshape(-1, 3) / N
    plan.close()
    xyz_g, _ = trace_paths(backend, fs, np.repeat(np.arange(W * H), N), np.tile(np.arange(N), W * H))
    g = xyz_g.astype(np.float64).reshape(W * H, N, 3)
    assert np.allclose(mg, g.mean(axis=1), rtol=1e-3, atol=1e-6)
    mo, so = oracle_moments(oracle, fs.to_abi(), W * H, N, N)
    for c, axis in enumerate("XYZ"):
        z = z_components(mo[:, c], so[:, c], mg[:, c], g[:, :, c].var(axis=1, ddof=1) / N)
        ok, count, cluster = passes_z_criteria(z, W, H)
        assert ok, (name, axis, count, cluster)


def test_device_entry_reads_device_arrays_only(exact_backend):
    """ix_accumulate_device on the carved, frosted stone under the sun: a scene whose
    finishes and tools are still host arrays declines before any launch; with every
    array in device memory it returns the host entry's sums."""
    import ctypes as C

    import torch

    from indicatrix_b200 import abi, workloads

    fs = workloads.carved_sun_frame(24, 20)
    n = fs.width * fs.height * 3
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = fs.to_abi()
    planes = torch.from_numpy(np.ascontiguousarray(fs.planes, np.float32)).cuda()
    sc.planes = C.cast(C.c_void_p(planes.data_ptr()), C.POINTER(C.c_float))
    assert exact_backend.accumulate_device(sc, 0, 8, out.data_ptr()) != 0
    fin = torch.from_numpy(np.ascontiguousarray(fs.facet_finishes, np.uint8)).cuda()
    sc.facet_finishes = C.cast(C.c_void_p(fin.data_ptr()), C.POINTER(C.c_uint8))
    raw = np.frombuffer(bytes((abi.Tool * len(fs.tools))(*fs.tools)), np.uint8).copy()
    tools = torch.from_numpy(raw).cuda()
    sc.tools = C.cast(C.c_void_p(tools.data_ptr()), C.POINTER(abi.Tool))
    assert exact_backend.accumulate_device(sc, 0, 8, out.data_ptr()) == 0
    torch.cuda.synchronize()
    acc = np.zeros((fs.height, fs.width, 3))
    assert exact_backend.try_accumulate(fs, 0, 8, acc)
    assert np.allclose(out.cpu().numpy().reshape(acc.shape), acc, rtol=1e-12, atol=1e-12)
