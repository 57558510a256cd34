"""The surrogate MLP's FP64 restatement (oracle/mlp_oracle.py), checked by central finite
differences so it can serve as the device gradients' checker; and the design-space helpers
of indicatrix_b200/surrogate.py (no GPU)."""
import numpy as np

import mlp_oracle as mo
from indicatrix_b200 import surrogate


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    dims = [5, 16, 16, 27]
    ws = [rng.standard_normal((a, b)) * 0.5 for a, b in zip(dims[:-1], dims[1:])]
    bs = [rng.standard_normal(b) * 0.1 for b in dims[1:]]
    x = rng.standard_normal((12, 5))
    t = rng.standard_normal((12, 27))
    # Without bf16 rounding the restatement is exact backprop: compare to differences.
    orig = mo.bf16
    mo.bf16 = lambda v: np.asarray(v, np.float64)
    try:
        _, grads = mo.gradients(ws, bs, x, t)
        eps = 1e-6
        for li in range(3):
            for (i, j) in [(0, 0), (1, 2), (3, 4)]:
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


def test_bf16_rounding_is_round_to_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.01171875, 3.0e-5, -2.5, 65504.0], np.float32)
    r = mo.bf16(vals)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[4] == -2.5


def test_design_box_and_normalisation():
    d = surrogate.sample_designs(100, 1)
    assert np.all(d >= surrogate.LOWER) and np.all(d <= surrogate.UPPER)
    z = surrogate.normalize(d)
    assert z.dtype == np.float32 and np.all(np.abs(z) <= 1.0)
    planes, disp = surrogate.design_stone(d[0])
    assert planes.shape[0] <= 128 and planes.shape[1] == 4
