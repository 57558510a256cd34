"""Parity of carved (concave-tool) stones on a B200 with the CPU oracle, through the C ABI.

The oracle's tool geometry and carve are pinned by the reference's own tests
(test_tools.py).  On the device the tool intervals and the carve run with every
operation rounded individually in both builds, so the boundary a ray meets is the
oracle's: per path in the exact build (isotropic, uniaxial and biaxial materials, sharp
and rounded edges), frame sums through the accumulate entry with the tools passed as the
call's argument or carried by the scene, batches equal to single calls, the white
furnace, and Tier 3 of the benched build on the reference harness's concave image
comparison ("Diamond, concave (table dimple + crown groove)", 48 x 48 px, 500 spp per
side, gpu_harness_last_run.json:79).
"""
import numpy as np
import pytest

from indicatrix_b200 import materials, workloads
from indicatrix_b200.backend import BatchPlan

from test_gpu_fast_parity import TIER3_H, TIER3_SPP, TIER3_W, oracle_moments, passes_z_criteria, z_components
from test_gpu_parity import trace_paths
from test_tools import carved_round_brilliant_tools

pytestmark = pytest.mark.gpu


def carved_frame(material, w=40, h=40, rounding=0.0, max_bounces=24):
    fs = workloads.round_brilliant_frame(w, h, max_bounces=max_bounces)
    fs.material = material
    if rounding:
        fs.material.edge_rounding_radius = rounding
    fs.tools = carved_round_brilliant_tools()
    return fs


CASES = {
    "diamond": lambda: materials.diamond(),
    "sapphire_tilted": lambda: materials.sapphire((0.0, 0.8, 0.6)),
    "tanzanite": lambda: materials.tanzanite((0.3, 0.8, 0.52)),
}


@pytest.mark.parametrize("rounding", [0.0, 0.02], ids=["sharp", "rounded"])
@pytest.mark.parametrize("name", list(CASES))
def test_carved_paths_match_oracle(exact_backend, oracle, name, rounding):
    """Per-path XYZ on identical (pixel, sample) inputs, the exact build: >= 99 % within
    1e-4, >= 85 % bit-identical, bounce counts equal on >= 98 % (the uniaxial bars)."""
    fs = carved_frame(CASES[name](), rounding=rounding)
    n, spp = fs.width * fs.height, 12
    xyz_o, bounces_o = oracle.trace_samples(fs.to_abi(), 0, n, 0, spp)
    xyz_g, bounces_g = trace_paths(exact_backend, fs, np.repeat(np.arange(n), spp), np.tile(np.arange(spp), n))
    xo = xyz_o.reshape(-1, 3).astype(np.float64)
    xg = xyz_g.astype(np.float64)
    rel = np.abs(xg - xo).max(axis=1) / np.maximum(np.abs(xo).max(axis=1), 1e-3)
    identical = np.all(xyz_g.view(np.uint32) == xyz_o.reshape(-1, 3).view(np.uint32), axis=1)
    stats = (np.mean(rel <= 1e-4), np.mean(identical), np.mean(bounces_g == bounces_o.ravel()))
    assert stats[0] >= 0.99 and stats[1] >= 0.85 and stats[2] >= 0.98, stats
    # the carve is exercised: the same frame without tools differs
    plain = carved_frame(CASES[name](), rounding=rounding)
    plain.tools = None
    xyz_p, _ = trace_paths(exact_backend, plain, np.repeat(np.arange(n), spp), np.tile(np.arange(spp), n))
    assert not np.array_equal(xyz_p, xyz_g)


def test_carved_frame_sums_and_the_tools_argument(exact_backend, oracle):
    """ix_accumulate_f64 on a carved stone: the per-pixel sums agree with the oracle's,
    and passing the tools as the call's argument equals the scene carrying them."""
    fs = carved_frame(materials.diamond(), 40, 32)
    acc = np.zeros((32, 40, 3))
    assert exact_backend.try_accumulate(fs, 0, 32, acc)
    _, s64, dropped = oracle.trace_frame(fs.to_abi(), 0, 32)
    assert dropped == 0
    rel = (np.abs(acc - s64) / np.maximum(np.abs(s64).max(axis=2, keepdims=True), 1e-3)).max(axis=2)
    assert np.mean(rel <= 1e-4) >= 0.95
    assert abs(acc.sum() - s64.sum()) / s64.sum() < 5e-3
    bare = carved_frame(materials.diamond(), 40, 32)
    tools = bare.tools
    bare.tools = None
    acc2 = np.zeros((32, 40, 3))
    assert exact_backend.try_accumulate_cancellable(bare, 0, 32, acc2, None, tools) == 0
    assert np.array_equal(acc, acc2)


def test_carved_batch_equals_single_calls(exact_backend):
    """A batch plan mixing a carved and a convex stone (one extended-instantiation launch)
    returns each scene's single-call sums bit for bit."""
    jobs = [(carved_frame(materials.diamond(), 24, 20), 0, 16),
            (workloads.round_brilliant_frame(24, 20), 3, 16),
            (carved_frame(materials.peridot(), 24, 20), 1, 16)]
    plan = BatchPlan(exact_backend, jobs)
    plan.run()
    for j, (fs, off, spp) in enumerate(jobs):
        single = np.zeros((20, 24, 3))
        assert exact_backend.try_accumulate(fs, off, spp, single)
        assert np.array_equal(plan.sums(j), single), j
    plan.close()


def test_carved_white_furnace_on_gpu(backend, oracle):
    """The oracle's carved furnace (test_tools) on the device, fast build: within 0.025
    of the dome's radiance."""
    from test_frosted import furnace_scene, furnace_target
    from indicatrix_b200.backend import FrameScene

    mat = materials.isotropic(materials.cauchy(1.5, 0.0, 0.0))
    sc, keep = furnace_scene(oracle, mat, finishes=False)
    planes = keep[0]
    fs = FrameScene(sc.camera, 12, 12, planes, mat, 12, sc.environment)
    fs.tools = carved_round_brilliant_tools()
    acc = np.zeros((12, 12, 3))
    assert backend.try_accumulate(fs, 0, 96, acc)
    mean = acc.reshape(-1, 3).sum(axis=0) / (12 * 12 * 96)
    target = furnace_target(oracle)
    assert np.all(np.abs(mean - target) / target <= 0.025), (mean, target)


def test_carved_tier3_fast_build(backend, oracle):
    """Tier 3 on the benched build for the reference harness's concave diamond: the batch
    plan's means over samples [0, 500) against the oracle's [500, 1000), each side's own
    variance (the device's from the per-path kernel over the same samples); the
    reference's rule on X, Y and Z."""
    W, H, N = TIER3_W, TIER3_H, TIER3_SPP
    fs = carved_frame(materials.diamond(), W, H)
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
        assert ok, (axis, count, cluster)
