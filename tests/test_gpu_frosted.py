"""Frosted (bruted) facets on a B200 through the C ABI against the CPU oracle:
apply_frosted_bounce (optics/raytracer/scattering/frosted.rs:289) in both transport
instantiations, and the reference's frosted-girdle furnace anchors
(material_equivalence_finish.rs:156, white_furnace_energy_conservation.rs:190).

The diffuse lobe's direction goes through sin/cos of (2 pi) u2, which the device and the
host libm round a few ULP apart, so a frosted path matches the oracle to that precision
rather than bit for bit; everything else on the path is as in test_gpu_parity.
"""
import numpy as np
import pytest

from indicatrix_b200 import materials
from indicatrix_b200.backend import FrameScene, GpuBatchItem, environment_preset, environment_uniform

from test_frosted import L0, bruted_girdle_finishes, furnace_target
from test_gpu_parity import trace_paths

pytestmark = pytest.mark.gpu


def girdle_scene(oracle, material, width=48, height=48, pitch=0.05, max_bounces=32, env=None):
    """The standard round brilliant with a bruted girdle, seen nearly edge-on."""
    planes = np.ascontiguousarray(oracle.standard_round_brilliant())
    cam = oracle.camera_new(0.4, pitch, 2.2, 30.0)
    env = env if env is not None else environment_preset(10, 1.0, 0.85, 0.95)
    return FrameScene(cam, width, height, planes, material, max_bounces, env,
                      bruted_girdle_finishes(planes.shape[0]))


@pytest.mark.parametrize("name", ["diamond", "sapphire"])
def test_frosted_paths_match_oracle(exact_backend, oracle, name):
    """Per path on identical (pixel, sample) inputs, exact build: >= 99 % within 1e-3
    relative and within 1e-2, the same bounce count on >= 98 %, the total within 1 %.
    (A path whose lobe angle rounds differently leaves in a different direction; on
    the sapphire stone 0.6 % of the paths do.)"""
    mat = materials.diamond() if name == "diamond" else materials.sapphire()
    fs = girdle_scene(oracle, mat)
    n = fs.width * fs.height
    xyz_o, bounces_o = oracle.trace_samples(fs.to_abi(), 0, n, 0, 8)
    xyz_g, bounces_g = trace_paths(exact_backend, fs, np.repeat(np.arange(n), 8), np.tile(np.arange(8), n))
    xo = xyz_o.reshape(-1, 3).astype(np.float64)
    xg = xyz_g.astype(np.float64)
    rel = np.abs(xg - xo).max(axis=1) / np.maximum(np.abs(xo).max(axis=1), 1e-3)
    stats = (np.mean(rel <= 1e-3), np.mean(rel <= 1e-2), np.mean(bounces_g == bounces_o.ravel()))
    assert stats[0] >= 0.99 and stats[1] >= 0.99 and stats[2] >= 0.98, stats
    assert abs(xg.sum() - xo.sum()) <= 1e-2 * xo.sum()


def test_frosted_frame_differs_from_polished(backend, oracle):
    """The girdle's finish reaches the device: the same frame with the girdle polished
    gives different sums, the frosted one agrees with the oracle's frame."""
    fs = girdle_scene(oracle, materials.diamond(), 32, 32)
    frosted = np.zeros((32, 32, 3))
    assert backend.try_accumulate(fs, 0, 32, frosted)
    fs.facet_finishes = None
    polished = np.zeros((32, 32, 3))
    assert backend.try_accumulate(fs, 0, 32, polished)
    assert not np.allclose(frosted, polished, rtol=1e-3)
    fs2 = girdle_scene(oracle, materials.diamond(), 32, 32)
    _, s64, _ = oracle.trace_frame(fs2.to_abi(), 0, 32)
    assert abs(frosted.sum() - s64.sum()) <= 2e-2 * s64.sum()


@pytest.mark.parametrize("birefringent", [False, True], ids=["isotropic", "birefringent"])
def test_frosted_girdle_furnace_on_gpu(backend, oracle, birefringent):
    """The frosted-girdle furnaces on the device (isotropic and uniaxial instantiations):
    the stone returns the uniform environment's radiance within 0.025 (depth 12)."""
    disp = materials.cauchy(1.5, 0.0, 0.0)
    mat = materials.uniaxial(disp, 0.03) if birefringent else materials.isotropic(disp)
    planes = np.ascontiguousarray(oracle.standard_round_brilliant())
    cam = oracle.camera_new(0.35, 0.28, 5.0, 18.0)
    fs = FrameScene(cam, 12, 12, planes, mat, 12, environment_uniform(L0), bruted_girdle_finishes(74))
    accum = np.zeros((12, 12, 3))
    assert backend.try_accumulate(fs, 0, 1024, accum)
    mean = accum.reshape(-1, 3).sum(0) / (12 * 12 * 1024)
    target = furnace_target(oracle)
    assert np.all(np.abs(mean - target) / target <= 0.025), (mean, target)


def test_frosted_batch_matches_single_calls(exact_backend, oracle):
    """Frosted and polished scenes in one batched launch give each scene's single-call
    sums bit for bit (the batch packs every scene's finishes)."""
    scenes = [girdle_scene(oracle, materials.diamond(), 24, 24),
              girdle_scene(oracle, materials.sapphire(), 24, 24, pitch=0.3)]
    plain = girdle_scene(oracle, materials.diamond(), 24, 24, pitch=0.6)
    plain.facet_finishes = None
    scenes.append(plain)
    singles = []
    for fs in scenes:
        a = np.zeros((24, 24, 3))
        assert exact_backend.try_accumulate(fs, 3, 16, a)
        singles.append(a)
    accs = [np.zeros((24, 24, 3)) for _ in scenes]
    items = [GpuBatchItem(fs, 3, 16, a) for fs, a in zip(scenes, accs)]
    assert exact_backend.try_accumulate_batch_cancellable(items) == 0
    for a, s in zip(accs, singles):
        assert np.array_equal(a.view(np.uint64), s.view(np.uint64))
