"""The surrogate MLP's FP64 restatement (oracle/mlp_oracle.py), checked by central finite
differences so it can serve as the device gradients' checker; and the design-space helpers
of indicatrix_b200/surrogate.py and include/ix_design.h that run on the host (no GPU)."""
import math

import numpy as np

import mlp_oracle as mo
from indicatrix_b200 import abi, geometry, surrogate


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    dims = [12, 16, 16, 27]
    ws = [rng.standard_normal((b, a)) * 0.5 for a, b in zip(dims[:-1], dims[1:])]
    bs = [rng.standard_normal(b) * 0.1 for b in dims[1:]]
    x = rng.standard_normal((12, 12))
    t = rng.standard_normal((12, 27))
    # Without bf16 rounding the restatement is exact backprop: compare to differences.
    orig = mo.bf16
    mo.bf16 = lambda v: np.asarray(v, np.float64)
    try:
        _, grads = mo.gradients(ws, bs, x, t)
        eps = 1e-6
        for li in range(3):
            for (i, j) in [(0, 0), (1, 2), (3, 4), (15, 11)]:
                if i >= ws[li].shape[0] or j >= ws[li].shape[1]:
                    continue
                wp = [w.copy() for w in ws]
                wm = [w.copy() for w in ws]
                wp[li][i, j] += eps
                wm[li][i, j] -= eps
                num = (mo.gradients(wp, bs, x, t)[0] - mo.gradients(wm, bs, x, t)[0]) / (2 * eps)
                assert abs(num - grads[li][0][i, j]) <= 1e-6 + 1e-4 * abs(num)
            bp = [b.copy() for b in bs]
            bm = [b.copy() for b in bs]
            bp[li][1] += eps
            bm[li][1] -= eps
            num = (mo.gradients(ws, bp, x, t)[0] - mo.gradients(ws, bm, x, t)[0]) / (2 * eps)
            assert abs(num - grads[li][1][1]) <= 1e-6 + 1e-4 * abs(num)
    finally:
        mo.bf16 = orig


def test_silu_derivative_matches_differences():
    z = np.linspace(-8.0, 8.0, 101)
    num = (mo.silu(z + 1e-6) - mo.silu(z - 1e-6)) / 2e-6
    assert np.max(np.abs(num - mo.silu_grad(z))) < 1e-8


def test_bf16_rounding_is_round_to_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.01171875, 3.0e-5, -2.5, 65504.0], np.float32)
    r = mo.bf16(vals)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[4] == -2.5


def test_design_box_and_normalisation():
    d = surrogate.sample_designs(100, 1)
    assert d.shape == (100, 12)
    assert np.all(d >= surrogate.LOWER) and np.all(d <= surrogate.UPPER)
    z = surrogate.normalize(d)
    assert z.dtype == np.float32 and np.all(np.abs(z) <= 1.0)
    assert len(surrogate.PARAM_NAMES) == 12 and surrogate.N_OUTPUTS == 27
    assert surrogate.DIMS == (12, 256, 256, 256, 27)


def test_design_planes_match_the_python_builder():
    """ix_design_planes (host C++) gives the planes of geometry.round_brilliant for the same
    parameters, to an f32 ulp (the two evaluate the same double formulas)."""
    for row in surrogate.sample_designs(20, 5):
        got = surrogate.design_planes(row, 64)
        p = geometry.RoundBrilliantParams(
            table_pct=float(np.float32(row[5])), crown_deg=float(np.float32(row[0])),
            pavilion_deg=float(np.float32(row[1])), girdle_pct=float(np.float32(row[6])),
            star_offset_deg=float(np.float32(row[2])), upper_half_offset_deg=float(np.float32(row[3])),
            lower_half_offset_deg=float(np.float32(row[4])))
        want = geometry.to_f32(geometry.round_brilliant(p))
        assert got.shape == want.shape == (121, 4)
        assert np.all(np.abs(got - want) <= 2.0 * np.spacing(np.abs(want).astype(np.float32)) + 1e-12)


def test_design_planes_reject_out_of_domain():
    row = surrogate.sample_designs(1, 2)[0].copy()
    row[0] = 95.0  # crown angle past vertical
    lib = surrogate._lib()
    r = np.ascontiguousarray(row, np.float32)
    assert lib.ix_design_planes(r.ctypes.data, 64, None, 0) == 0
    row = surrogate.sample_designs(1, 2)[0].copy()
    row[7] = math.nan
    r = np.ascontiguousarray(row, np.float32)
    assert lib.ix_design_planes(r.ctypes.data, 64, None, 0) == 0


def test_design_material_is_cauchy_through_nd_and_dispersion():
    row = surrogate.sample_designs(1, 3)[0].copy()
    row[9] = 2.0
    m = surrogate.design_material(row)
    assert m.dispersion.kind == abi.DISP_CAUCHY
    A, B = m.dispersion.b[0], m.dispersion.b[1]
    n = lambda l_um: A + B / (l_um * l_um)  # noqa: E731
    assert abs(n(0.5893) - np.float32(row[7])) < 1e-5
    assert abs((n(0.4861) - n(0.6563)) - np.float32(row[8])) < 1e-5
    assert m.abs_o.n_bands == 1 and m.abs_e.n_bands == 1
    assert abs(m.abs_o.bands[0].peak - 2.0) < 1e-6 and m.abs_o.bands[0].shape == abi.BAND_GAUSS_WAVELENGTH
    row[9] = 0.0
    assert surrogate.design_material(row).abs_o.n_bands == 0


def test_offspring_stay_in_the_box_and_keep_parents():
    rng = np.random.default_rng(0)
    parents = surrogate.sample_designs(8, 4)
    kids = surrogate._offspring(rng, parents, 100, 0.3)
    assert kids.shape == (100, 12)
    assert np.all(kids >= surrogate.LOWER) and np.all(kids <= surrogate.UPPER)
    assert np.array_equal(kids[:8], parents)


def test_score_weighs_metrics_by_scale():
    m = np.zeros((2, 27))
    m[0, :9] = 2.0   # brilliance
    m[1, 9:18] = 1.0  # fire
    s = surrogate.score(m, np.array([2.0, 0.5, 1.0]))
    assert np.allclose(s, [1.0, 2.0])


def _analytic_metrics(d):
    """A smooth stand-in for the tracer on the design box: [n, 27], maximal at the box's
    centre in every normalised parameter."""
    z = surrogate.normalize(d).astype(np.float64)
    base = 1.0 - 0.1 * (z ** 2).sum(axis=1)
    tilt = np.linspace(1.0, 0.8, 9)
    return np.concatenate([np.outer(base, tilt), 0.1 * np.outer(base, tilt), 0.5 * np.outer(base, tilt)], axis=1)


class _FakeEnsemble:
    """Members that agree except on designs with a large first parameter."""

    def __init__(self, noise):
        self.noise = noise

    def score(self, x, scales):
        d = surrogate.LOWER + (np.asarray(x, np.float64) + 1.0) / 2.0 * (surrogate.UPPER - surrogate.LOWER)
        m = _analytic_metrics(d)
        s = surrogate.score(m, scales)
        dis = np.where(x[:, 0] > 0.8, self.noise, 0.0)
        return m, s, dis


def test_traced_search_improves_and_counts_every_candidate():
    calls = []

    def evaluate(d):
        calls.append(len(d))
        return _analytic_metrics(d)

    scales = np.array([1.0, 0.1, 0.5])
    cfg = surrogate.SearchConfig(population=256, generations=6, elite=16, seed=3)
    r = surrogate.traced_search(None, scales, cfg, evaluate=evaluate)
    assert r.evaluations == 256 * 6 and r.traced == 256 * 6 and calls == [256] * 6
    assert all(b >= a for a, b in zip(r.history, r.history[1:]))  # elitist: never worse
    assert r.history[-1] > r.history[0]
    assert np.all(r.best_design >= surrogate.LOWER) and np.all(r.best_design <= surrogate.UPPER)


def test_screened_search_falls_back_on_disagreement_and_retraces_the_elite():
    traced = []

    def evaluate(d):
        traced.append(np.array(d))
        return _analytic_metrics(d)

    scales = np.array([1.0, 0.1, 0.5])
    cfg = surrogate.SearchConfig(population=256, generations=4, elite=16, fallback=0.02, seed=5)
    r = surrogate.screened_search(None, _FakeEnsemble(0.05), scales, cfg, evaluate=evaluate)
    assert r.evaluations == 256 * 4
    # Every candidate over the disagreement bar went to the tracer, and the elite of each
    # generation was re-rendered (those already traced as fallbacks are not traced twice).
    assert r.fallbacks > 0 and r.traced == sum(len(t) for t in traced)
    assert r.traced <= r.fallbacks + 16 * 4
    for t in traced:
        assert len(t) > 0
    # With members that always agree nothing falls back and only the elite is traced.
    traced.clear()
    r2 = surrogate.screened_search(None, _FakeEnsemble(0.0), scales, cfg, evaluate=evaluate)
    assert r2.fallbacks == 0 and r2.traced == 16 * 4
    assert r2.history[-1] >= r2.history[0]
    # The best design's reported metrics are traced ones.
    assert np.allclose(r2.best_metrics, _analytic_metrics(r2.best_design[None])[0])
