"""The analytic optical metrics (brilliance, fire, scintillation, windowing, extinction;
color/metrics/evaluate.rs) on a B200 against the CPU oracle, through the C ABI.

The fan traces use only IEEE-exact arithmetic (no transcendental until the fire angle's
acos), so in the exact-rounding build the ray classification -- and with it brilliance,
windowing, extinction and scintillation -- reproduces the oracle bit for bit; fire
differs by the device acos's last bits.
"""
import math

import numpy as np
import pytest

from indicatrix_b200 import geometry, materials, workloads
from indicatrix_b200.backend import MetricsLighting

from test_gpu_parity import ulp_diff
from test_oracle_golden import GOLDEN_METRICS

pytestmark = pytest.mark.gpu


def test_golden_metrics_on_gpu(exact_backend, oracle):
    """golden_regression.rs:210-233 on the device."""
    planes = oracle.standard_round_brilliant()
    got = exact_backend.evaluate_gem_optical_metrics(planes, materials.diamond(), 0.0, 0.45,
                                                     MetricsLighting(10, 0.85, 0.95))
    want = np.array(GOLDEN_METRICS, np.uint32).view(np.float32)
    d = ulp_diff(got, want)
    assert d[0] == 0 and d[2] == 0 and d[3] == 0 and d[4] == 0, (got, want)
    assert d[1] <= 64, (got, want)


def metric_cases():
    stones = [(geometry.to_f32(geometry.round_brilliant()), materials.diamond()),
              (geometry.to_f32(geometry.step_cut()), materials.sapphire())]
    for st in workloads.random_stones(3, seed=17):
        stones.append((st.planes, st.material))
    poses = []
    for s in range(len(stones)):
        for yaw, pitch in [(0.0, math.pi / 2), (0.6, 0.45), (2.0, 1.1), (4.0, 0.8)]:
            poses.append((s, np.float32(yaw), np.float32(pitch)))
    return stones, poses


@pytest.mark.parametrize("lighting", [MetricsLighting(10, 0.85, 0.95), MetricsLighting(1, 0.0, 0.0, 16.0),
                                      MetricsLighting(1, 0.0, 0.0, 30.0), MetricsLighting(8, 2.1, 0.4)],
                         ids=["ring", "iso16", "iso30", "incandescent"])
def test_metrics_batch_matches_oracle(exact_backend, backend, oracle, lighting):
    """Many stones x poses in one launch: exact build identical to the oracle except the
    fire index (a few ULP); fused build within a few classified rays."""
    stones, poses = metric_cases()
    got = exact_backend.evaluate_metrics_batch([(p, m.dispersion) for p, m in stones], poses, lighting)
    fast = backend.evaluate_metrics_batch([(p, m.dispersion) for p, m in stones], poses, lighting)
    for i, (s, yaw, pitch) in enumerate(poses):
        planes, mat = stones[s]
        want = oracle.metrics(planes, mat, float(yaw), float(pitch), lighting.preset, lighting.light_yaw,
                              lighting.light_pitch, lighting.head_shadow_deg)
        d = ulp_diff(got[i], want)
        assert d[0] == 0 and d[2] == 0 and d[3] == 0 and d[4] == 0, (i, got[i], want)
        assert d[1] <= 256 or abs(got[i][1] - want[1]) <= 1e-4 * max(want[1], 1.0), (i, got[i], want)
        # Fused rounding can flip a ray's classification; the fire index rests on the few
        # rays whose n_F and n_C traces leave by the same facet, so one flip moves it most.
        tol = np.maximum(1.5, 0.02 * np.abs(want))
        tol[1] = max(6.0, 0.15 * abs(want[1]))
        assert np.all(np.abs(fast[i] - want) <= tol), (i, fast[i], want)


def test_metrics_consumed_only(backend, oracle):
    """MetricsWanted::CONSUMED_ONLY: fire and scintillation report the placeholders and
    the other three equal the full evaluation's."""
    stones, poses = metric_cases()
    lighting = MetricsLighting(10, 0.85, 0.95)
    full = backend.evaluate_metrics_batch([(p, m.dispersion) for p, m in stones], poses, lighting)
    core = backend.evaluate_metrics_batch([(p, m.dispersion) for p, m in stones], poses, lighting,
                                          want_fire_and_scintillation=False)
    assert np.all(core[:, 1] == 25.0) and np.all(core[:, 2] == 75.0)
    assert np.array_equal(core[:, [0, 3, 4]], full[:, [0, 3, 4]])
