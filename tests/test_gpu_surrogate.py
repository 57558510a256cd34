"""The surrogate on the device: the tcgen05 BF16 GEMM and its fused epilogues against FP64
numpy on the same bf16-rounded operands, the MLP's gradients against the FP64 oracle
(oracle/mlp_oracle.py), and the traced design metrics (include/ix_design.h)."""
import numpy as np
import pytest

import mlp_oracle as mo
from indicatrix_b200 import surrogate

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda().to(dtype)


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


# FP32 accumulation of k bf16 products against the exact FP64 sum: a relative bound on the
# sum of |products| that grows with k.
def _tol(k):
    return 2e-6 * max(4.0, np.sqrt(k))


@pytest.mark.parametrize("shape", [(128, 64, 64), (70, 37, 29), (256, 128, 5), (5, 27, 128), (1, 1, 1),
                                   (300, 200, 100), (4096, 256, 256), (256, 256, 4096), (27, 256, 4096),
                                   (4096, 27, 256), (129, 257, 1000)])
def test_gemm_bf16_matches_fp64(shape):
    import torch

    m, n, k = shape
    rng = np.random.default_rng(m * n + k)
    for ta in (0, 1):
        for tb in (0, 1):
            a = rng.standard_normal((k, m) if ta else (m, k)).astype(np.float32)
            b = rng.standard_normal((n, k) if tb else (k, n)).astype(np.float32)
            ad, bd = _dev(a, torch.bfloat16), _dev(b, torch.bfloat16)
            c = torch.full((m, n), np.nan, dtype=torch.float32, device="cuda")
            rc = surrogate._lib().ix_mlp_gemm_bf16(ta, tb, m, n, k, ad.data_ptr(), a.shape[1], bd.data_ptr(),
                                                   b.shape[1], c.data_ptr(), n, _stream())
            assert rc == 0
            A = mo.bf16(a).T if ta else mo.bf16(a)
            B = mo.bf16(b).T if tb else mo.bf16(b)
            want = A @ B
            got = c.cpu().numpy()
            scale = np.abs(A) @ np.abs(B) + 1e-30
            err = np.abs(got - want) / scale
            assert np.all(np.isfinite(got)), (ta, tb)
            assert err.max() <= _tol(k), (ta, tb, err.max())
    assert surrogate._lib().ix_mlp_status(1) == 0


def test_gemm_strided_output_leaves_padding():
    """ldc > n: the columns between n and ldc are not written."""
    import torch

    m, n, k, ldc = 130, 40, 70, 48
    rng = np.random.default_rng(1)
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((k, n)).astype(np.float32)
    c = torch.full((m, ldc), -7.0, dtype=torch.float32, device="cuda")
    assert surrogate._lib().ix_mlp_gemm_bf16(0, 0, m, n, k, _dev(a, torch.bfloat16).data_ptr(), k,
                                             _dev(b, torch.bfloat16).data_ptr(), n, c.data_ptr(), ldc,
                                             _stream()) == 0
    got = c.cpu().numpy()
    assert np.all(got[:, n:] == -7.0)
    want = mo.bf16(a) @ mo.bf16(b)
    assert np.max(np.abs(got[:, :n] - want) / (np.abs(mo.bf16(a)) @ np.abs(mo.bf16(b)))) <= _tol(k)


@pytest.mark.parametrize("m,n,k", [(4096, 256, 256), (100, 27, 256), (33, 256, 12)])
def test_linear_epilogue_bias_silu(m, n, k):
    import torch

    rng = np.random.default_rng(m + n + k)
    x = rng.standard_normal((m, k)).astype(np.float32)
    w = (rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32)
    bias = rng.standard_normal(n).astype(np.float32)
    z = torch.empty(m, n, dtype=torch.float32, device="cuda")
    h = torch.empty(m, n, dtype=torch.float32, device="cuda")
    hb = torch.empty(m, n, dtype=torch.bfloat16, device="cuda")
    bd = torch.from_numpy(bias).cuda()
    assert surrogate._lib().ix_mlp_linear(m, n, k, _dev(x, torch.bfloat16).data_ptr(), k,
                                          _dev(w, torch.bfloat16).data_ptr(), bd.data_ptr(), 1, z.data_ptr(),
                                          h.data_ptr(), hb.data_ptr(), _stream()) == 0
    X, W = mo.bf16(x), mo.bf16(w)
    want_z = X @ W.T + bias
    scale = np.abs(X) @ np.abs(W).T + np.abs(bias) + 1e-30
    zd = z.cpu().numpy()
    assert np.max(np.abs(zd - want_z) / scale) <= _tol(k)
    hd = h.cpu().numpy()
    # SiLU of the device's own z, to the fast exponential's accuracy.
    assert np.max(np.abs(hd - mo.silu(zd.astype(np.float64))) / (1.0 + np.abs(zd))) <= 2e-6
    # The bf16 copy is the device's f32 h rounded to nearest even.
    assert np.array_equal(hb.float().cpu().numpy(), mo.bf16(hd).astype(np.float32))


def test_backward_silu_epilogue():
    import torch

    m, n, k = 512, 256, 256  # dz_next m x k, W k x n, z_prev m x n
    rng = np.random.default_rng(5)
    dzn = rng.standard_normal((m, k)).astype(np.float32)
    w = (rng.standard_normal((k, n)) / 16.0).astype(np.float32)
    zp = rng.standard_normal((m, n)).astype(np.float32) * 3.0
    dz = torch.empty(m, n, dtype=torch.float32, device="cuda")
    dzb = torch.empty(m, n, dtype=torch.bfloat16, device="cuda")
    assert surrogate._lib().ix_mlp_backward_silu(m, n, k, _dev(dzn, torch.bfloat16).data_ptr(),
                                                 _dev(w, torch.bfloat16).data_ptr(),
                                                 torch.from_numpy(zp).cuda().data_ptr(), dz.data_ptr(),
                                                 dzb.data_ptr(), _stream()) == 0
    g = mo.bf16(dzn) @ mo.bf16(w)
    sg = mo.silu_grad(zp.astype(np.float64))
    want = g * sg
    ab = np.abs(mo.bf16(dzn)) @ np.abs(mo.bf16(w))
    got = dz.cpu().numpy()
    # The GEMM's accumulation error scaled by |silu'|, plus the fast logistic's absolute
    # error in silu' (a few 1e-7; silu' crosses zero near z = -1.28) times |dz_next W|.
    bound = _tol(k) * ab * np.abs(sg) + 2e-6 * ab
    assert np.all(np.abs(got - want) <= bound), np.max(np.abs(got - want) / bound)
    assert np.array_equal(dzb.float().cpu().numpy(), mo.bf16(got).astype(np.float32))


@pytest.mark.parametrize("dims,batch", [((12, 64, 64, 27), 96), (surrogate.DIMS, 512)])
def test_mlp_gradients_match_fp64_oracle(dims, batch):
    net = surrogate.SurrogateMLP(dims, seed=4)
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, (batch, dims[0])).astype(np.float32)
    t = rng.standard_normal((batch, dims[-1])).astype(np.float32)
    loss, grads = net.gradients(x, t)
    ws = [L.w.cpu().numpy().astype(np.float64) for L in net.layers]
    bs = [L.b.cpu().numpy().astype(np.float64) for L in net.layers]
    loss_o, grads_o = mo.gradients(ws, bs, x, t)
    assert abs(float(loss.item()) - loss_o) <= 1e-4 * loss_o
    for (dw, db), (dw_o, db_o) in zip(grads, grads_o):
        dw, db = dw.cpu().numpy(), db.cpu().numpy()
        assert dw.shape == dw_o.shape
        # bf16 rounding of the device's own intermediate activations differs from the
        # oracle's where an f32 value sits at a rounding boundary: a relative bound.
        assert np.linalg.norm(dw - dw_o) <= 1e-2 * np.linalg.norm(dw_o)
        assert np.linalg.norm(db - db_o) <= 1e-2 * np.linalg.norm(db_o)
    assert surrogate._lib().ix_mlp_status(1) == 0


def test_training_reduces_the_loss():
    net = surrogate.SurrogateMLP(seed=2)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (4096, 12)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, i % 12]) + 0.5 * x[:, (i + 3) % 12] ** 2 for i in range(27)], axis=1)
    losses = net.fit(x, t.astype(np.float32), epochs=60, batch=512, lr=2e-3)
    assert losses[-1] < 0.05 * losses[0], (losses[0], losses[-1])


def test_design_metrics_are_deterministic_and_in_range(backend):
    d = surrogate.sample_designs(6, 21)
    spec = surrogate.RenderSpec(width=32, height=32, spp=16)
    a = surrogate.evaluate_designs(backend, d, spec)
    b = surrogate.evaluate_designs(backend, d, spec)
    assert a.shape == (6, 27)
    assert np.array_equal(a, b)
    assert np.all(np.isfinite(a))
    bri, fire, sci = a[:, :9], a[:, 9:18], a[:, 18:]
    assert np.all(bri > 0.0) and np.all(bri < 2.0)
    assert np.all(fire >= 0.0) and np.all(fire < 0.5)
    assert np.all(sci > 0.0) and np.all(sci < 5.0)
    # Chunked calls give the same metrics as one call (each job's sample range is its own).
    c = surrogate.evaluate_designs(backend, d, spec, max_per_call=4)
    assert np.array_equal(a, c)


def test_split_half_metrics_converge_without_noise_bias(backend):
    """Metrics at 64 spp and at 1024 spp (disjoint samples) agree closely on average: the
    split-half estimators carry no per-pixel noise bias."""
    d = surrogate.sample_designs(16, 22)
    lo = surrogate.evaluate_designs(backend, d, surrogate.RenderSpec(spp=64, sample_offset=0))
    hi = surrogate.evaluate_designs(backend, d, surrogate.RenderSpec(spp=1024, sample_offset=64))
    tl, th = surrogate.tilt_means(lo), surrogate.tilt_means(hi)
    rel = (tl - th) / th
    # Mean relative deviation per metric across designs: no systematic offset.
    assert np.all(np.abs(rel.mean(axis=0)) < 0.03), rel.mean(axis=0)


def test_surrogate_screened_search_against_tracer_only_search(backend):
    """Config 5 at reduced scale: the 4-member ensemble, trained on traced designs, screens
    an evolutionary search (population 4096, top 64 re-traced per generation, tracer
    fallback above 2 % ensemble disagreement) against the same search scored by the tracer
    alone, both timed the same way (host designs in, host metrics out).  The screened
    search must deliver >= 20x the design evaluations per second, its final design's
    metrics must be within 1 % of that design's 1024-spp render, and its final design must
    score within 3 % of the tracer-only search's (the ensemble is refined on the designs the
    search traces, as the search goes)."""
    spec = surrogate.RenderSpec(width=32, height=32, spp=64)
    train = surrogate.sample_designs(16384, 31)
    y = surrogate.evaluate_designs(backend, train, spec)
    scales = surrogate.tilt_means(y).mean(axis=0)
    ens = surrogate.SurrogateEnsemble(4, seed=3)
    ens.fit(surrogate.normalize(train), y, epochs=300, batch=4096, lr=1e-3)
    hold = surrogate.sample_designs(256, 32)
    y_hold = surrogate.evaluate_designs(backend, hold, surrogate.RenderSpec(spp=1024, sample_offset=1 << 20))
    _, s_hold, dis = ens.score(surrogate.normalize(hold), scales)
    s_true = surrogate.score(y_hold, scales)
    assert np.median(np.abs(s_hold - s_true) / s_true) < 0.05
    assert np.mean(dis > 0.02) < 0.05
    cfg = surrogate.SearchConfig(population=4096, generations=6, elite=64, fallback=0.02, seed=7)
    screened = surrogate.screened_search(backend, ens, scales, cfg, spec)
    traced = surrogate.traced_search(backend, scales, cfg, spec)
    assert screened.evaluations == traced.evaluations == 4096 * 6
    assert screened.evals_per_s >= 20.0 * traced.evals_per_s, (screened.evals_per_s, traced.evals_per_s)
    final = surrogate.evaluate_designs(backend, np.stack([screened.best_design, traced.best_design]),
                                       surrogate.RenderSpec(spp=1024, sample_offset=1 << 21))
    err = surrogate.relative_error(screened.best_metrics, final[0])
    assert np.all(err <= 0.01), err
    f = surrogate.score(final, scales)
    assert f[0] >= 0.97 * f[1], f
