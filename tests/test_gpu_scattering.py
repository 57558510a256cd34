"""Henyey-Greenstein interior scattering on the device (uniaxial instantiation, which also
traces isotropic stones) against the
CPU oracle: per-path parity on identical samples (exact build; the HG azimuth goes through
sin / cos and the free flight through log, which device and host libm round a few ULP
apart), the reference's scattering furnaces, batch == single calls."""
import numpy as np
import pytest

from indicatrix_b200 import materials, workloads
from indicatrix_b200.backend import GpuBatchItem

from test_frosted import furnace_target
from test_gpu_frosted import girdle_scene
from test_gpu_parity import trace_paths

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [("diamond", 1.2, 0.4), ("diamond", 4.0, 0.8), ("diamond", 2.0, -0.3),
                                  ("sapphire", 1.5, 0.5)])
def test_scattering_paths_match_oracle(exact_backend, oracle, case):
    name, sigma_s, g = case
    fs = workloads.round_brilliant_frame(48, 48, 32)
    base = materials.diamond() if name == "diamond" else materials.sapphire()
    fs.material = materials.with_scattering(base, sigma_s, g)
    n = fs.width * fs.height
    xyz_o, bounces_o = oracle.trace_samples(fs.to_abi(), 0, n, 0, 8)
    xyz_g, bounces_g = trace_paths(exact_backend, fs, np.repeat(np.arange(n), 8), np.tile(np.arange(8), n))
    xo = xyz_o.reshape(-1, 3).astype(np.float64)
    xg = xyz_g.astype(np.float64)
    rel = np.abs(xg - xo).max(axis=1) / np.maximum(np.abs(xo).max(axis=1), 1e-3)
    stats = (np.mean(rel <= 1e-3), np.mean(rel <= 1e-2), np.mean(bounces_g == bounces_o.ravel()))
    assert stats[0] >= 0.98 and stats[1] >= 0.98 and stats[2] >= 0.97, stats
    assert abs(xg.sum() - xo.sum()) <= 2e-2 * xo.sum()


@pytest.mark.parametrize("case", ["lossless", "dispersive"])
def test_scattering_furnaces_on_gpu(backend, oracle, case):
    from indicatrix_b200.backend import FrameScene, environment_uniform

    from test_frosted import L0

    if case == "lossless":
        mat, depth, tol = materials.with_scattering(materials.isotropic(materials.cauchy(1.5, 0.0, 0.0)), 1.2, 0.4), 16, 0.03
    else:
        mat, depth, tol = materials.with_scattering(materials.diamond(), 1.5, 0.3), 64, 0.02
    planes = np.ascontiguousarray(oracle.standard_round_brilliant())
    cam = oracle.camera_new(0.35, 0.28, 5.0, 18.0)
    fs = FrameScene(cam, 12, 12, planes, mat, depth, environment_uniform(L0))
    acc = np.zeros((12, 12, 3))
    assert backend.try_accumulate(fs, 0, 4096, acc)
    mean = acc.reshape(-1, 3).sum(0) / (12 * 12 * 4096)
    target = furnace_target(oracle)
    assert np.all(np.abs(mean - target) / target <= tol), (mean, target)


def test_scattering_batch_matches_single_calls(exact_backend, oracle):
    scenes = []
    for sg, pitch in (((1.2, 0.4), 0.05), ((3.0, -0.2), 0.3)):
        fs = girdle_scene(oracle, materials.with_scattering(materials.diamond(), *sg), 24, 24, pitch=pitch)
        scenes.append(fs)
    plain = workloads.round_brilliant_frame(24, 24)
    scenes.append(plain)
    singles = []
    for fs in scenes:
        a = np.zeros((24, 24, 3))
        assert exact_backend.try_accumulate(fs, 1, 16, a)
        singles.append(a)
    accs = [np.zeros((24, 24, 3)) for _ in scenes]
    assert exact_backend.try_accumulate_batch_cancellable([GpuBatchItem(fs, 1, 16, a) for fs, a in zip(scenes, accs)]) == 0
    for a, s in zip(accs, singles):
        assert np.array_equal(a.view(np.uint64), s.view(np.uint64))


@pytest.mark.parametrize("name", ["diamond", "sapphire"])
def test_rounded_edges_paths_match_oracle(exact_backend, oracle, name):
    """Rounded facet edges (shading_normal_near_edge, intersect.rs:196) on the device,
    per path against the oracle on identical samples (exact build), and the frame differs
    from the sharp-edged one."""
    fs = workloads.round_brilliant_frame(48, 48, 32)
    fs.material = materials.diamond() if name == "diamond" else materials.sapphire()
    fs.material.edge_rounding_radius = 0.03
    n = fs.width * fs.height
    xyz_o, bounces_o = oracle.trace_samples(fs.to_abi(), 0, n, 0, 8)
    xyz_g, bounces_g = trace_paths(exact_backend, fs, np.repeat(np.arange(n), 8), np.tile(np.arange(8), n))
    xo = xyz_o.reshape(-1, 3).astype(np.float64)
    xg = xyz_g.astype(np.float64)
    rel = np.abs(xg - xo).max(axis=1) / np.maximum(np.abs(xo).max(axis=1), 1e-3)
    stats = (np.mean(rel <= 1e-3), np.mean(rel <= 1e-2), np.mean(bounces_g == bounces_o.ravel()))
    assert stats[0] >= 0.98 and stats[1] >= 0.99 and stats[2] >= 0.98, stats
    sharp = workloads.round_brilliant_frame(48, 48, 32)
    sharp.material = materials.diamond() if name == "diamond" else materials.sapphire()
    a, b = np.zeros((48, 48, 3)), np.zeros((48, 48, 3))
    assert exact_backend.try_accumulate(fs, 0, 8, a) and exact_backend.try_accumulate(sharp, 0, 8, b)
    assert not np.allclose(a, b, rtol=1e-3)
