"""Every lighting model on a B200 against the CPU oracle, through the C ABI.

The oracle's lookup reproduces the reference's 180 environment pins (test_environment).
On the device: the escape radiance of all 15 presets per function (CHECK_ENV, both
builds); the reference's own pin hashes recomputed from the exact build's values for the
presets whose spectra take no exponential (D65 and the wavelength-free geometry); per-path
parity of the exact build on the diamond under every model the path traces; Tier 3 of the
benched build under the tent and the sun.
"""
import ctypes as C

import numpy as np
import pytest

from indicatrix_b200 import materials, workloads
from indicatrix_b200.backend import BatchPlan

from test_environment import FNV_OFFSET, GOLDEN, fold, pin_directions, rows
from test_gpu_fast_parity import TIER3_H, TIER3_SPP, TIER3_W, oracle_moments, passes_z_criteria, ulp_diff, z_components
from test_gpu_parity import CHECK_ENV, small_scene, trace_paths

pytestmark = pytest.mark.gpu

# Presets whose radiance takes no exponential: D65 studio, iso-hemisphere, the D65 tents,
# the dome and the sun.
NO_EXP = (1, 2, 3, 4, 5, 6, 7)
NEW_MODELS = (0, 2, 3, 4, 5, 6, 12)


def oracle_env(oracle, env, inp):
    f32p = oracle._f32p
    return np.array([oracle.lib().ixo_environment_channel(C.byref(env), f32p(r[:3].copy()), float(r[3]),
                                                          f32p(r[4:7].copy())) for r in inp], np.float32)


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_every_preset_per_function(backend, exact_backend, oracle, exact):
    """CHECK_ENV on 1500 random (direction, wavelength, observer) rows per preset and pose,
    with a tray: within 4 ULP in the exact build (CUDA's expf in the blackbody, band and
    line spectra), within the reference's sample_studio_environment budget (8192 ULP,
    floor 1e-6) in the fast build."""
    b = exact_backend if exact else backend
    rng = np.random.default_rng(5)
    fs = small_scene()
    for preset in range(15):
        for yaw, pitch, tray in [(0.84, 0.94, 0.0), (-2.1, 0.3, 0.3)]:
            env = oracle.environment_preset(preset, 1.3, yaw, pitch, tray, 1.0, 16.0)
            fs.environment = env
            d = rng.normal(size=(1500, 3)).astype(np.float32)
            obs = rng.normal(size=(1500, 3)).astype(np.float32)
            obs /= np.linalg.norm(obs, axis=1, keepdims=True)
            lam = rng.uniform(380, 780, (1500, 1)).astype(np.float32)
            inp = np.concatenate([d, lam, obs], axis=1).astype(np.float32)
            out = b.debug_check(fs, CHECK_ENV, inp, 1).view(np.float32)[:, 0]
            want = oracle_env(oracle, env, inp)
            u = ulp_diff(out, want)
            floor = np.abs(out.astype(np.float64) - want) < 1e-6
            assert np.all((u <= (4 if exact else 8192)) | floor), (preset, int(u.max()))


def test_reference_pins_on_the_device(exact_backend, oracle):
    """as_lit_is_bit_identical's rows recomputed from the exact build's device values: the
    reference's own hashes for every preset whose radiance takes no exponential."""
    fs = small_scene()
    dirs = pin_directions()
    for idx, pose, obs, shadow, pin in rows():
        if idx not in NO_EXP:
            continue
        fs.environment = oracle.environment_preset(idx, GOLDEN["exposure"], pose[0], pose[1], 0.0, 1.0, shadow)
        inp = np.array([[*d, lam, *obs] for d in dirs for lam in GOLDEN["lambdas"]], np.float32)
        out = exact_backend.debug_check(fs, CHECK_ENV, inp, 1).view(np.uint32)[:, 0]
        h = FNV_OFFSET
        for v in out:
            h = fold(h, v)
        assert h == pin, (GOLDEN["presets"][idx], pose, shadow)


@pytest.mark.parametrize("preset", NEW_MODELS)
def test_new_models_paths_match_oracle(exact_backend, oracle, preset):
    """Per-path XYZ of the exact build, the diamond under each model past the studio rig
    and the iso-hemisphere (tent, white tray, shop, window, dome, sun, ASET): >= 99 % of
    paths within 1e-4 of the oracle, bounce counts equal on >= 98 %."""
    fs = workloads.round_brilliant_frame(40, 40)
    fs.environment = oracle.environment_preset(preset, 1.0, 0.84, 0.94)
    n, spp = fs.width * fs.height, 8
    xyz_o, bounces_o = oracle.trace_samples(fs.to_abi(), 0, n, 0, spp)
    xyz_g, bounces_g = trace_paths(exact_backend, fs, np.repeat(np.arange(n), spp), np.tile(np.arange(spp), n))
    xo = xyz_o.reshape(-1, 3).astype(np.float64)
    rel = np.abs(xyz_g - xo).max(axis=1) / np.maximum(np.abs(xo).max(axis=1), 1e-3)
    stats = (np.mean(rel <= 1e-4), np.mean(bounces_g == bounces_o.ravel()))
    assert stats[0] >= 0.99 and stats[1] >= 0.98, (preset, stats)


@pytest.mark.parametrize("preset", [0, 6])
def test_new_models_tier3_fast_build(backend, oracle, preset):
    """Tier 3 on the benched build under the light tent and the sun: the batch plan's
    means over [0, 500) against the oracle's [500, 1000), each side's own variance."""
    W, H, N = TIER3_W, TIER3_H, TIER3_SPP
    fs = workloads.round_brilliant_frame(W, H)
    fs.environment = oracle.environment_preset(preset, 1.0, 0.84, 0.94)
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
        assert ok, (preset, axis, count, cluster)
