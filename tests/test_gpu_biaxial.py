"""Parity of the biaxial transport on a B200 with the CPU oracle, through the C ABI.

The oracle's biaxial indicatrix is pinned by the reference's own biaxial tests
(test_biaxial.py).  Here the device is checked against it: per function in both rounding
builds, to the reference harness's Tier-2 budgets (ULP or absolute floor,
renderer/gpu/transport_check/eigenmodes_biaxial/*.rs: wave_indices 64 / 1e-5,
eigen_polarizations 48 / 5e-5, mode_poynting_dir 48 / 1e-5, resolve_entry_mode 4096,
assigned-mode alpha 1200 / 1e-5); per path in the exact build on the four biaxial
built-ins; and by the Tier-3 statistics (z_stats.rs:95-110) of the benched fast build on
the reference harness's biaxial image comparisons (Alexandrite, Topaz, Tanzanite; 48 x 48
px, 500 spp per side, gpu_harness_last_run.json:82-86).
"""
import ctypes as C

import numpy as np
import pytest

from indicatrix_b200 import materials, workloads
from indicatrix_b200.backend import BatchPlan

from test_gpu_fast_parity import (TIER3_H, TIER3_SPP, TIER3_W, oracle_moments, passes_z_criteria, ulp_diff,
                                  within, z_components)
from test_gpu_parity import trace_paths

pytestmark = pytest.mark.gpu

CHECK_BIAXIAL = 17
BIAXIAL = ("alexandrite", "topaz", "tanzanite", "peridot")
# (name, output columns, ULP budget, absolute floor)
FIELDS = [("wave_indices", slice(0, 2), 64, 1e-5),
          ("eigen_polarizations", slice(2, 8), 48, 5e-5),
          ("mode_poynting_dir", slice(8, 14), 48, 1e-5),
          ("resolve_entry_mode", slice(14, 22), 4096, 1e-5),
          ("assigned_mode_alpha", slice(22, 24), 1200, 1e-5)]


def frame_with(material, w=16, h=16, max_bounces=24):
    fs = workloads.round_brilliant_frame(w, h, max_bounces=max_bounces)
    fs.material = material
    return fs


def check_inputs(oracle, m, n, seed):
    """Random incident wave normals against random facet normals (cos_i = -k . n > 0),
    wavelengths over the visible range and the material's n_beta there (the oracle's
    dispersion: the indicatrix functions are checked on their own, as the reference's
    harness checks them from given principal indices)."""
    rng = np.random.default_rng(seed)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    k = rng.normal(size=(n, 3))
    k /= np.linalg.norm(k, axis=1, keepdims=True)
    flip = np.sum(k * nrm, axis=1) > 0
    k[flip] = -k[flip]
    k = k.astype(np.float32)
    nrm = nrm.astype(np.float32)
    k = (k / np.sqrt(np.sum(k * k, axis=1, keepdims=True))).astype(np.float32)
    cos_i = np.clip(-np.sum(k.astype(np.float64) * nrm, axis=1), 0.0, 1.0).astype(np.float32)
    lam = rng.uniform(380.0, 780.0, size=n).astype(np.float32)
    nb = np.array([oracle.lib().ixo_dispersion_eval(C.byref(m.dispersion), C.c_float(x)) for x in lam], np.float32)
    return np.concatenate([k, nrm, cos_i[:, None], lam[:, None], nb[:, None]], axis=1).astype(np.float32)


def oracle_bundle(oracle, m, rows):
    out = np.zeros((rows.shape[0], 24), np.float32)
    f32p = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    for i, r in enumerate(rows):
        k = np.ascontiguousarray(r[0:3])
        nn = np.ascontiguousarray(r[3:6])
        o = np.zeros(24, np.float32)
        oracle.lib().ixo_biaxial_bundle(C.byref(m), f32p(k), f32p(nn), C.c_float(r[6]), C.c_float(r[7]),
                                        C.c_float(r[8]), f32p(o))
        out[i] = o
    return out


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
@pytest.mark.parametrize("name", BIAXIAL)
def test_biaxial_functions_match_oracle(backend, exact_backend, oracle, name, exact):
    """wave_indices, eigen_polarizations, mode_poynting_dir, resolve_entry_mode and the
    trichroic assigned-mode alpha of each channel's own indicatrix, 2048 random cases per
    material: every comparison within the reference's budget or floor in both builds.  The
    indicatrix functions round every operation individually in both builds, so both are
    bit-exact on them; the alpha is within 4 ULP in the exact build (its Gaussian bands
    take CUDA's expf against the host libm's)."""
    b = exact_backend if exact else backend
    m = getattr(materials, name)((0.3, 0.8, 0.52))
    rows = check_inputs(oracle, m, 2048, 17 + BIAXIAL.index(name))
    got = b.debug_check(frame_with(m), CHECK_BIAXIAL, rows, 24).view(np.float32)
    want = oracle_bundle(oracle, m, rows)
    assert np.all(np.isfinite(got))
    for field, cols, budget, floor in FIELDS:
        ok = within(got[:, cols], want[:, cols], budget, floor)
        assert np.all(ok), (field, int((~ok).sum()), np.argwhere(~ok)[:4].tolist())
    assert np.array_equal(got[:, :22].view(np.uint32), want[:, :22].view(np.uint32))
    if exact:
        assert ulp_diff(got[:, 22:], want[:, 22:]).max() <= 4


@pytest.mark.parametrize("name", BIAXIAL)
def test_biaxial_paths_match_oracle(exact_backend, oracle, name):
    """Per-path XYZ of the exact build on identical (pixel, sample) inputs, the optic axis
    tilted off the table normal: branch decisions follow the oracle's, so nearly every
    path carries the oracle's bits (bars as the uniaxial transport's: >= 99 % within 1e-4,
    >= 85 % bit-identical, bounce counts equal on >= 98 %)."""
    fs = frame_with(getattr(materials, name)((0.3, 0.8, 0.52)), 40, 40)
    n, spp = fs.width * fs.height, 12
    xyz_o, bounces_o = oracle.trace_samples(fs.to_abi(), 0, n, 0, spp)
    xyz_g, bounces_g = trace_paths(exact_backend, fs, np.repeat(np.arange(n), spp), np.tile(np.arange(spp), n))
    xo = xyz_o.reshape(-1, 3).astype(np.float64)
    xg = xyz_g.astype(np.float64)
    rel = np.abs(xg - xo).max(axis=1) / np.maximum(np.abs(xo).max(axis=1), 1e-3)
    identical = np.all(xyz_g.view(np.uint32) == xyz_o.reshape(-1, 3).view(np.uint32), axis=1)
    stats = (np.mean(rel <= 1e-4), np.mean(identical), np.mean(bounces_g == bounces_o.ravel()))
    assert stats[0] >= 0.99 and stats[1] >= 0.85 and stats[2] >= 0.98, stats
    assert abs(xg.sum() - xo.sum()) <= 1e-2 * xo.sum()


def test_biaxial_frame_sums_match_oracle(exact_backend, oracle):
    """The whole-frame entry (ix_accumulate_f64) on a biaxial stone: per-pixel sums of
    the same samples agree with the oracle's."""
    fs = frame_with(materials.tanzanite((0.3, 0.8, 0.52)), 40, 32)
    acc = np.zeros((32, 40, 3))
    assert exact_backend.try_accumulate(fs, 0, 32, acc)
    _, s64, dropped = oracle.trace_frame(fs.to_abi(), 0, 32)
    assert dropped == 0 and exact_backend.last_dropped() == 0
    rel = (np.abs(acc - s64) / np.maximum(np.abs(s64).max(axis=2, keepdims=True), 1e-3)).max(axis=2)
    assert np.mean(rel <= 1e-4) >= 0.95
    assert abs(acc.sum() - s64.sum()) / s64.sum() < 5e-3


@pytest.mark.parametrize("name", ["alexandrite", "topaz", "tanzanite"])
def test_biaxial_tier3_fast_build(backend, oracle, name):
    """Tier 3 on the benched build: a batch plan (one persistent launch, the kernel the
    frame and batch benchmarks time) traces samples [0, 500) of a 48 x 48 biaxial frame,
    the oracle samples [500, 1000); the reference's pass rule on X, Y and Z.  Each side's
    standard error is its own sample variance (z_stats.rs:11-80): the device's from the
    per-path check kernel over the same samples, whose per-pixel means the plan's sums
    reproduce.  (A bright, heavy-tailed stone such as Alexandrite needs this: one side's
    variance taken for both understates the error wherever that side missed a rare bright
    sample, and the rule then flags ~30 pixels of 2304.)"""
    W, H, N = TIER3_W, TIER3_H, TIER3_SPP
    fs = frame_with(getattr(materials, name)(), W, H)
    plan = BatchPlan(backend, [(fs, 0, N)])
    plan.run()
    mg = plan.sums(0).reshape(-1, 3) / N
    plan.close()
    xyz_g, _ = trace_paths(backend, fs, np.repeat(np.arange(W * H), N), np.tile(np.arange(N), W * H))
    g = xyz_g.astype(np.float64).reshape(W * H, N, 3)
    sg = g.var(axis=1, ddof=1) / N
    assert np.allclose(mg, g.mean(axis=1), rtol=1e-3, atol=1e-6)
    mo, so = oracle_moments(oracle, fs.to_abi(), W * H, N, N)
    for c, axis in enumerate("XYZ"):
        z = z_components(mo[:, c], so[:, c], mg[:, c], sg[:, c])
        ok, count, cluster = passes_z_criteria(z, W, H)
        assert ok, (name, axis, count, cluster)


def test_biaxial_batch_equals_single_calls(exact_backend):
    """A batch plan mixing a biaxial, a uniaxial and an isotropic scene returns each
    scene's single-call sums bit for bit in the exact build (one uniaxial-instantiation
    launch serves all three)."""
    backend = exact_backend
    jobs = [(frame_with(materials.peridot((0.3, 0.8, 0.52)), 24, 20), 0, 16),
            (frame_with(materials.sapphire(), 24, 20), 5, 16),
            (frame_with(materials.diamond(), 24, 20), 0, 16)]
    plan = BatchPlan(backend, jobs)
    plan.run()
    for j, (fs, off, spp) in enumerate(jobs):
        single = np.zeros((20, 24, 3))
        assert backend.try_accumulate(fs, off, spp, single)
        assert np.array_equal(plan.sums(j), single), j
    plan.close()
