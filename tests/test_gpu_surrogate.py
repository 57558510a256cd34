"""The surrogate on the device: the BF16 tensor-core GEMM against FP64 numpy, the MLP's
gradients against the FP64 oracle (oracle/mlp_oracle.py), and what the trained network
gains: held-out accuracy, and a screened search that finds better designs than the same
number of metric evaluations spent on random candidates, at a far higher rate of
candidates scored per second."""
import time

import numpy as np
import pytest

import mlp_oracle as mo
from indicatrix_b200 import surrogate

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(64, 64, 16), (70, 37, 29), (256, 128, 5), (5, 27, 128), (1, 1, 1)])
def test_gemm_bf16_matches_fp64(shape):
    import torch

    m, n, k = shape
    rng = np.random.default_rng(m * n + k)
    for ta in (0, 1):
        for tb in (0, 1):
            a = rng.standard_normal((k, m) if ta else (m, k)).astype(np.float32)
            b = rng.standard_normal((n, k) if tb else (k, n)).astype(np.float32)
            ad = torch.from_numpy(a).cuda().to(torch.bfloat16)
            bd = torch.from_numpy(b).cuda().to(torch.bfloat16)
            c = torch.full((m, n), np.nan, dtype=torch.float32, device="cuda")
            rc = surrogate._lib().ix_mlp_gemm_bf16(ta, tb, m, n, k, ad.data_ptr(), a.shape[1], bd.data_ptr(),
                                                   b.shape[1], c.data_ptr(), n,
                                                   torch.cuda.current_stream().cuda_stream)
            assert rc == 0
            A = mo.bf16(a).T if ta else mo.bf16(a)
            B = mo.bf16(b).T if tb else mo.bf16(b)
            want = A @ B
            got = c.cpu().numpy()
            scale = np.abs(A) @ np.abs(B) + 1e-30
            assert np.all(np.abs(got - want) <= 1e-5 * scale), (ta, tb)


def test_mlp_gradients_match_fp64_oracle():
    net = surrogate.SurrogateMLP(hidden=64, seed=4)
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, (96, surrogate.N_FEATURES)).astype(np.float32)
    t = rng.uniform(0, 1, (96, surrogate.N_OUTPUTS)).astype(np.float32)
    loss, grads = net.gradients(x, t)
    ws = [L.w.cpu().numpy() for L in net.layers]
    bs = [L.b.cpu().numpy() for L in net.layers]
    loss_o, grads_o = mo.gradients(ws, bs, x, t)
    assert abs(loss - loss_o) <= 1e-4 * loss_o
    for (dw, db), (dw_o, db_o) in zip(grads, grads_o):
        dw, db = dw.cpu().numpy(), db.cpu().numpy()
        assert np.linalg.norm(dw - dw_o) <= 2e-2 * np.linalg.norm(dw_o)
        assert np.linalg.norm(db - db_o) <= 2e-2 * np.linalg.norm(db_o)


def test_trained_surrogate_screens_designs(backend):
    train_d = surrogate.sample_designs(3072, 11)
    test_d = surrogate.sample_designs(512, 12)
    t0 = time.perf_counter()
    train_y = surrogate.evaluate_designs(backend, train_d)
    eval_rate = len(train_d) / (time.perf_counter() - t0)
    test_y = surrogate.evaluate_designs(backend, test_d)
    net = surrogate.SurrogateMLP(hidden=128, seed=1)
    losses = net.fit(surrogate.normalize(train_d), train_y, epochs=120, batch=256, lr=2e-3)
    assert losses[-1] < 0.5 * losses[0]  # on standardised targets
    pred = net.predict(surrogate.normalize(test_d))
    mse = np.mean((pred - test_y) ** 2)
    base = np.mean((test_y.mean(axis=0) - test_y) ** 2)  # predicting the mean: no network
    assert mse < 0.25 * base, (mse, base)
    # Per output, on the outputs that vary across designs: R^2 well above 0.
    var = test_y.var(axis=0)
    live = var > 1e-6 * var.max()
    r2 = 1.0 - ((pred - test_y) ** 2).mean(axis=0)[live] / var[live]
    assert np.median(r2) > 0.5, r2
    # Screening: 8192 candidates ranked by the network, the best 64 re-evaluated; the
    # same 64 metric evaluations spent on random candidates find a worse best design.
    cands = surrogate.sample_designs(8192, 13)
    t0 = time.perf_counter()
    net.predict(surrogate.normalize(cands))
    screen_rate = len(cands) / (time.perf_counter() - t0)
    best_d, best_y = surrogate.screened_search(backend, net, cands, 64)
    rand_y = surrogate.evaluate_designs(backend, surrogate.sample_designs(64, 14))
    assert surrogate.score(best_y)[0] >= surrogate.score(rand_y).max()
    assert screen_rate > 5 * eval_rate, (screen_rate, eval_rate)
