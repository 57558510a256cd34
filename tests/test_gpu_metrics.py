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
                                      MetricsLighting(1, 0.0, 0.0, 30.0), MetricsLighting(8, 2.1, 0.4),
                                      MetricsLighting(0, 0.85, 0.95), MetricsLighting(3, 0.4, 1.0, 20.0),
                                      MetricsLighting(5, 0.85, 0.95), MetricsLighting(6, 0.4, 0.9),
                                      MetricsLighting(13, 0.85, 0.95)],
                         ids=["ring", "iso16", "iso30", "incandescent", "tent", "shop", "dome", "sun", "uv365"])
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


def to_radians(deg):
    """f32::to_radians: deg * (PI / 180), the constant rounded to f32 first."""
    return np.float32(np.float32(deg) * np.float32(np.float32(np.pi) / np.float32(180.0)))


def tilt_slot(job):
    """tilt_slot (color/metrics/pose_batch.rs:117)."""
    half = 90
    if job == 0:
        return half
    return 2 * half - (job - 1) if job <= half else job - 1 - half


def test_tilt_slots_cover_the_axis():
    """pose_batch.rs tests: every_pose_lands_in_its_own_tilt_slot."""
    slots = [tilt_slot(j) for j in range(181)]
    assert sorted(slots) == list(range(181))
    assert (tilt_slot(0), tilt_slot(1), tilt_slot(91), tilt_slot(90), tilt_slot(180)) == (90, 180, 0, 91, 89)


def test_angular_profile_matches_oracle(exact_backend, oracle):
    """evaluate_angular_profile_at_azimuth (profile.rs:37): the 19 elevations of
    PROFILE_ANGLES_DEG, each curve point bit-identical to the oracle's pose."""
    planes = oracle.standard_round_brilliant()
    light = MetricsLighting(10, 0.85, 0.95)
    b, e, w = exact_backend.evaluate_angular_profile_at_azimuth(planes, materials.diamond(), 0.3, light)
    for i in range(19):
        want = oracle.metrics(planes, materials.diamond(), 0.3, float(to_radians(5.0 * i)), 10, 0.85, 0.95)
        assert ulp_diff([b[i], e[i], w[i]], [want[0], want[4], want[3]]).max() == 0, i


def test_all_axes_profiles_match_oracle(exact_backend, backend, oracle):
    """evaluate_all_axes_profiles (sweep.rs:74): 4 azimuths x 181 tilts in one launch.
    Exact build: every point bit-identical to the oracle's pose at axis_poses'
    (yaw, pitch), placed by tilt_slot; fast build: within a few classified rays."""
    planes = geometry.to_f32(geometry.step_cut())
    mat = materials.sapphire()
    light = MetricsLighting(1, 0.0, 0.0, 16.0)
    got = exact_backend.evaluate_all_axes_profiles(planes, mat, light)
    fast = backend.evaluate_all_axes_profiles(planes, mat, light)
    assert len(got) == 4 and len(fast) == 4
    for a, az in enumerate([0.0, 45.0, 90.0, 135.0]):
        positive, negative = to_radians(az), to_radians(np.float32(az) + np.float32(180.0))
        poses = [(positive, to_radians(90.0))] + [(positive, to_radians(i)) for i in range(90)] + \
                [(negative, to_radians(i)) for i in range(90)]
        for job in range(0, 181, 7):
            yaw, pitch = poses[job]
            want = oracle.metrics(planes, mat, float(yaw), float(pitch), 1, 0.0, 0.0, 16.0)
            s = tilt_slot(job)
            g = [got[a].brilliance[s], got[a].extinction[s], got[a].windowing[s]]
            assert ulp_diff(g, [want[0], want[4], want[3]]).max() == 0, (a, job)
            f = np.array([fast[a].brilliance[s], fast[a].extinction[s], fast[a].windowing[s]])
            w3 = np.array([want[0], want[4], want[3]])
            assert np.all(np.abs(f - w3) <= np.maximum(1.5, 0.02 * np.abs(w3))), (a, job, f, want)


def test_aset_scores_as_the_iso_hemisphere(exact_backend):
    """scoring_preset (color/metrics/lighting.rs:125): the ASET view is a false-colour
    diagnostic, scored as the grading standard, so switching to it never moves the numbers."""
    stones, poses = metric_cases()
    args = [(p, m.dispersion) for p, m in stones]
    aset = exact_backend.evaluate_metrics_batch(args, poses, MetricsLighting(12, 0.3, 0.7, 20.0))
    iso = exact_backend.evaluate_metrics_batch(args, poses, MetricsLighting(1, 0.3, 0.7, 20.0))
    assert np.array_equal(np.asarray(aset), np.asarray(iso))
