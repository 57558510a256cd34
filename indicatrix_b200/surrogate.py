"""Learned surrogate for design search: an MLP from a round brilliant's design parameters
(table %, crown and pavilion angles, refractive index, dispersion) to its tilt-resolved
brilliance / fire / scintillation, trained on metrics this library computes on the GPU
(``GpuBackend.evaluate_metrics_batch``, the reference's evaluate_gem_optical_metrics),
with forward, backward and Adam on the library's own kernels (``include/ix_surrogate.h``:
BF16 tensor-core GEMM with FP32 accumulation).  ``screened_search`` ranks many candidate
designs with the network and re-evaluates only the best with the metrics kernel.

No reference counterpart (the reference optimizes on the analytic metrics directly).
torch provides device memory and the stream; every arithmetic step runs in the library.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import geometry, materials
from .backend import GpuBackend, MetricsLighting, load_library

TILTS_DEG = [0.0, 5.0, 10.0, 15.0, 20.0, 25.0, 30.0, 35.0, 40.0]
N_FEATURES = 5
N_OUTPUTS = 3 * len(TILTS_DEG)  # brilliance, fire, scintillation at each tilt
# Design space: table %, crown deg, pavilion deg, n_d, dispersion (Cauchy B in um^2).
LOWER = np.array([45.0, 25.0, 37.0, 1.5, 0.002], np.float64)
UPPER = np.array([70.0, 45.0, 45.0, 2.5, 0.02], np.float64)

_bound = False


def _lib() -> C.CDLL:
    global _bound
    lib = load_library()
    if not _bound:
        vp, f32p = C.c_void_p, C.POINTER(C.c_float)
        u32, u64, f32 = C.c_uint32, C.c_uint64, C.c_float
        lib.ix_mlp_gemm_bf16.argtypes = [C.c_int, C.c_int, u32, u32, u32, vp, u32, vp, u32, vp, u32, vp]
        lib.ix_mlp_bias_act.argtypes = [u32, u32, vp, vp, C.c_int, vp, vp, vp, vp]
        lib.ix_mlp_mse_grad.argtypes = [u32, u32, vp, vp, vp, vp, vp, vp]
        lib.ix_mlp_relu_backward.argtypes = [u64, vp, vp, vp, vp, vp]
        lib.ix_mlp_bias_grad.argtypes = [u32, u32, vp, vp, vp]
        lib.ix_mlp_adam.argtypes = [u64, vp, vp, vp, vp, vp, f32, f32, f32, f32, u32, vp]
        lib.ix_mlp_to_bf16.argtypes = [u64, vp, vp, vp]
        del f32p
        _bound = True
    return lib


def _ok(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("surrogate kernel launch failed")


# ---- designs and their metrics --------------------------------------------------------
def sample_designs(n: int, seed: int) -> np.ndarray:
    """n designs uniform over the design box, [n, 5]."""
    rng = np.random.default_rng(seed)
    return LOWER + (UPPER - LOWER) * rng.random((n, N_FEATURES))


def normalize(designs: np.ndarray) -> np.ndarray:
    return ((designs - LOWER) / (UPPER - LOWER) * 2.0 - 1.0).astype(np.float32)


def design_stone(d: np.ndarray) -> Tuple[np.ndarray, object]:
    planes = geometry.to_f32(geometry.round_brilliant(geometry.RoundBrilliantParams(
        table_pct=float(d[0]), crown_deg=float(d[1]), pavilion_deg=float(d[2]))))
    return planes, materials.cauchy(float(d[3]), float(d[4]), 0.0)


def evaluate_designs(backend: GpuBackend, designs: np.ndarray,
                     lighting: Optional[MetricsLighting] = None) -> np.ndarray:
    """The metrics kernel's brilliance, fire and scintillation of every design at every
    tilt in one launch: [n, 27] (brilliance % / 100, fire, scintillation % / 100)."""
    lighting = lighting if lighting is not None else MetricsLighting(10, 0.85, 0.95)
    stones = [design_stone(d) for d in designs]
    poses = [(i, 0.0, math.radians(90.0 - t)) for i in range(len(designs)) for t in TILTS_DEG]
    m = backend.evaluate_metrics_batch(stones, poses, lighting, True)
    if m is None:
        raise RuntimeError(f"metrics declined: {backend.last_lost_reason()}")
    m = m.reshape(len(designs), len(TILTS_DEG), 5)
    # GemOpticalMetrics order: brilliance %, fire index, scintillation %, windowing %, extinction %.
    out = np.concatenate([m[:, :, 0] / 100.0, m[:, :, 1], m[:, :, 2] / 100.0], axis=1)
    return out.astype(np.float32)


# ---- the network ----------------------------------------------------------------------
@dataclass
class Layer:
    w: object   # f32 [in, out] master weights (torch)
    wb: object  # bf16 copy
    b: object   # f32 [out]
    mw: object
    vw: object
    mb: object
    vb: object


class SurrogateMLP:
    """[5] -> hidden -> hidden -> [27], ReLU, MSE, Adam; BF16 GEMMs with FP32 accumulation
    on the library's tensor-core kernel, FP32 master weights."""

    def __init__(self, hidden: int = 128, seed: int = 0, device: str = "cuda") -> None:
        import torch

        self.torch = torch
        self.dev = torch.device(device)
        g = np.random.default_rng(seed)
        dims = [N_FEATURES, hidden, hidden, N_OUTPUTS]
        self.layers: List[Layer] = []
        for fan_in, fan_out in zip(dims[:-1], dims[1:]):
            w = torch.from_numpy((g.standard_normal((fan_in, fan_out)) * math.sqrt(2.0 / fan_in)).astype(np.float32))
            w = w.to(self.dev)
            z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=self.dev)  # noqa: E731
            layer = Layer(w, torch.empty(fan_in, fan_out, dtype=torch.bfloat16, device=self.dev), z(fan_out),
                          z(fan_in, fan_out), z(fan_in, fan_out), z(fan_out), z(fan_out))
            _ok(_lib().ix_mlp_to_bf16(w.numel(), w.data_ptr(), layer.wb.data_ptr(), self._stream()))
            self.layers.append(layer)
        self.step = 0
        # Per-output standardisation of the targets (set by fit): the outputs differ in
        # scale by orders of magnitude, and the loss weighs them equally once scaled.
        self.t_mean = np.zeros(N_OUTPUTS, np.float32)
        self.t_std = np.ones(N_OUTPUTS, np.float32)

    def _stream(self) -> int:
        return self.torch.cuda.current_stream().cuda_stream

    def _bf16(self, x):
        xb = self.torch.empty(x.shape, dtype=self.torch.bfloat16, device=self.dev)
        _ok(_lib().ix_mlp_to_bf16(x.numel(), x.data_ptr(), xb.data_ptr(), self._stream()))
        return xb

    def _forward(self, xb, m: int):
        """Returns per layer (input bf16, pre-activation z) and the f32 output."""
        torch, lib, s = self.torch, _lib(), self._stream()
        acts = []
        h = xb
        out = None
        for li, L in enumerate(self.layers):
            k, n = L.w.shape
            acc = torch.empty(m, n, dtype=torch.float32, device=self.dev)
            _ok(lib.ix_mlp_gemm_bf16(0, 0, m, n, k, h.data_ptr(), k, L.wb.data_ptr(), n, acc.data_ptr(), n, s))
            last = li == len(self.layers) - 1
            z = torch.empty_like(acc)
            if last:
                out = torch.empty_like(acc)
                _ok(lib.ix_mlp_bias_act(m, n, acc.data_ptr(), L.b.data_ptr(), 0, z.data_ptr(), out.data_ptr(), None, s))
                acts.append((h, z))
            else:
                hb = torch.empty(m, n, dtype=torch.bfloat16, device=self.dev)
                _ok(lib.ix_mlp_bias_act(m, n, acc.data_ptr(), L.b.data_ptr(), 1, z.data_ptr(), None, hb.data_ptr(), s))
                acts.append((h, z))
                h = hb
        return acts, out

    def predict(self, x: np.ndarray) -> np.ndarray:
        torch = self.torch
        xt = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(self.dev)
        _, out = self._forward(self._bf16(xt), x.shape[0])
        return out.cpu().numpy() * self.t_std + self.t_mean

    def gradients(self, x: np.ndarray, t: np.ndarray):
        """Loss and the f32 gradients [(dW, db) per layer] of one batch (no update)."""
        torch, lib, s = self.torch, _lib(), self._stream()
        m = x.shape[0]
        xt = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(self.dev)
        tt = torch.from_numpy(np.ascontiguousarray(t, np.float32)).to(self.dev)
        acts, out = self._forward(self._bf16(xt), m)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        dy = torch.empty_like(out)
        dyb = torch.empty(out.shape, dtype=torch.bfloat16, device=self.dev)
        _ok(lib.ix_mlp_mse_grad(m, out.shape[1], out.data_ptr(), tt.data_ptr(), dy.data_ptr(), dyb.data_ptr(),
                                loss.data_ptr(), s))
        grads = [None] * len(self.layers)
        d_f32, d_b16 = dy, dyb
        for li in range(len(self.layers) - 1, -1, -1):
            L = self.layers[li]
            h_in, _z = acts[li]
            k, n = L.w.shape
            dw = torch.empty(k, n, dtype=torch.float32, device=self.dev)
            # dW = h_in^T dZ  (h_in: m x k, dZ: m x n)
            _ok(lib.ix_mlp_gemm_bf16(1, 0, k, n, m, h_in.data_ptr(), k, d_b16.data_ptr(), n, dw.data_ptr(), n, s))
            db = torch.empty(n, dtype=torch.float32, device=self.dev)
            _ok(lib.ix_mlp_bias_grad(m, n, d_f32.data_ptr(), db.data_ptr(), s))
            grads[li] = (dw, db)
            if li > 0:
                # dH_prev = dZ W^T, then through the previous layer's ReLU.
                dh = torch.empty(m, k, dtype=torch.float32, device=self.dev)
                _ok(lib.ix_mlp_gemm_bf16(0, 1, m, k, n, d_b16.data_ptr(), n, L.wb.data_ptr(), n, dh.data_ptr(), k, s))
                z_prev = acts[li - 1][1]
                dz = torch.empty_like(dh)
                dzb = torch.empty(m, k, dtype=torch.bfloat16, device=self.dev)
                _ok(lib.ix_mlp_relu_backward(dh.numel(), dh.data_ptr(), z_prev.data_ptr(), dz.data_ptr(), dzb.data_ptr(),
                                             s))
                d_f32, d_b16 = dz, dzb
        return float(loss.item()), grads

    def train_step(self, x: np.ndarray, t: np.ndarray, lr: float = 2e-3) -> float:
        lib, s = _lib(), self._stream()
        loss, grads = self.gradients(x, t)
        self.step += 1
        for L, (dw, db) in zip(self.layers, grads):
            _ok(lib.ix_mlp_adam(L.w.numel(), L.w.data_ptr(), L.wb.data_ptr(), dw.data_ptr(), L.mw.data_ptr(),
                                L.vw.data_ptr(), lr, 0.9, 0.999, 1e-8, self.step, s))
            _ok(lib.ix_mlp_adam(L.b.numel(), L.b.data_ptr(), None, db.data_ptr(), L.mb.data_ptr(), L.vb.data_ptr(),
                                lr, 0.9, 0.999, 1e-8, self.step, s))
        return loss

    def fit(self, x: np.ndarray, t: np.ndarray, epochs: int = 200, batch: int = 256, lr: float = 2e-3,
            seed: int = 0) -> List[float]:
        rng = np.random.default_rng(seed)
        self.t_mean = t.mean(axis=0).astype(np.float32)
        self.t_std = np.maximum(t.std(axis=0), 1e-6).astype(np.float32)
        t = ((t - self.t_mean) / self.t_std).astype(np.float32)
        losses = []
        for _ in range(epochs):
            order = rng.permutation(x.shape[0])
            ep = []
            for i in range(0, x.shape[0], batch):
                idx = order[i:i + batch]
                ep.append(self.train_step(x[idx], t[idx], lr))
            losses.append(float(np.mean(ep)))
        return losses


def score(metrics: np.ndarray) -> np.ndarray:
    """A design's search score: mean over tilts of brilliance + fire + scintillation."""
    return metrics.reshape(metrics.shape[0], 3, len(TILTS_DEG)).mean(axis=2).sum(axis=1)


def screened_search(backend: GpuBackend, net: SurrogateMLP, candidates: np.ndarray, keep: int):
    """Rank `candidates` with the network, re-evaluate the best `keep` with the metrics
    kernel, return (designs, metrics) of the survivors in descending true score."""
    pred = net.predict(normalize(candidates))
    best = np.argsort(-score(pred))[:keep]
    true = evaluate_designs(backend, candidates[best])
    order = np.argsort(-score(true))
    return candidates[best][order], true[order]
