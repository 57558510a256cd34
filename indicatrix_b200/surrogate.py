"""Learned surrogate for design search over 12-parameter round brilliants.

* ``evaluate_designs`` renders designs with the batched path tracer and measures their
  brilliance / fire / scintillation at 9 tilts (``include/ix_design.h``: one persistent
  launch over designs x tilts, image metrics reduced on the device).
* ``SurrogateMLP`` is the 12 -> 256 -> 256 -> 256 -> 27 SiLU network, BF16 weights and
  activations with FP32 accumulation: forward, backward and Adam run on the library's
  kernels (``include/ix_surrogate.h``: tcgen05 GEMMs with fused bias / SiLU epilogues).
* ``SurrogateEnsemble`` trains several members from different seeds; their disagreement
  on a candidate's score decides whether the tracer must score it instead.
* ``screened_search`` is the evolutionary search in which the ensemble scores every
  candidate, candidates it disagrees on fall back to the tracer, and the tracer re-renders
  the best of each generation; ``traced_search`` is the same search scored by the tracer
  alone, the baseline it is measured against.

No reference counterpart: the reference's cut optimiser scores candidates with its
analytic metrics (crates/indicatrix-cut-core/src/optimize/mod.rs:1-80).  torch provides
device memory and the stream; every arithmetic step runs in the library.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import abi
from .backend import GpuBackend, camera_new, environment_preset, load_library, PRESET_ISO_HEMISPHERE

PARAM_NAMES = ("crown_deg", "pavilion_deg", "star_offset_deg", "upper_half_offset_deg", "lower_half_offset_deg",
               "table_pct", "girdle_pct", "n_d", "dispersion", "absorb_peak", "absorb_center_nm", "absorb_width_nm")
N_FEATURES = len(PARAM_NAMES)
# The design box: the batched workload's cut and material ranges (crown 25-45 deg,
# pavilion 37-45 deg, table 45-70 %, n_D 1.45-2.60, n_F - n_C 0.01-0.07, absorption
# 0-5 /cm) and the facet offsets and girdle of common round brilliants.
LOWER = np.array([25.0, 37.0, -16.0, 3.0, 0.5, 45.0, 1.0, 1.45, 0.01, 0.0, 420.0, 20.0], np.float64)
UPPER = np.array([45.0, 45.0, -8.0, 10.0, 3.0, 70.0, 4.0, 2.60, 0.07, 5.0, 680.0, 120.0], np.float64)
TILTS_DEG = (0.0, 5.0, 10.0, 15.0, 20.0, 25.0, 30.0, 35.0, 40.0)
METRICS = ("brilliance", "fire", "scintillation")
N_OUTPUTS = len(METRICS) * len(TILTS_DEG)  # output k = metric k // 9 at tilt k % 9
DIMS = (N_FEATURES, 256, 256, 256, N_OUTPUTS)
FACE_UP_DISTANCE = 1.6
FOV_DEG = 42.0

_bound = False
# Kernel launches this module has enqueued (the bench's launch count).
launches = 0


class DesignView(C.Structure):
    """ix_design_view (include/ix_design.h)."""
    _fields_ = [
        ("cameras", C.POINTER(abi.Camera)),
        ("n_views", C.c_uint32),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("spp", C.c_uint32),
        ("sample_offset", C.c_uint32),
        ("max_bounces", C.c_uint32),
        ("girdle_segments", C.c_uint32),
        ("environment", abi.Environment),
    ]


def _lib() -> C.CDLL:
    global _bound
    lib = load_library()
    if not _bound:
        vp = C.c_void_p
        u32, u64, f32 = C.c_uint32, C.c_uint64, C.c_float
        lib.ix_mlp_gemm_bf16.argtypes = [C.c_int, C.c_int, u32, u32, u32, vp, u32, vp, u32, vp, u32, vp]
        lib.ix_mlp_linear.argtypes = [u32, u32, u32, vp, u32, vp, vp, C.c_int, vp, vp, vp, vp]
        lib.ix_mlp_backward_silu.argtypes = [u32, u32, u32, vp, vp, vp, vp, vp, vp]
        lib.ix_mlp_status.argtypes = [C.c_int]
        lib.ix_mlp_status.restype = u32
        lib.ix_mlp_mse_grad.argtypes = [u32, u32, vp, vp, vp, vp, vp, vp]
        lib.ix_mlp_bias_grad.argtypes = [u32, u32, vp, vp, vp]
        lib.ix_mlp_adam.argtypes = [u64, vp, vp, vp, vp, vp, f32, f32, f32, f32, u32, vp]
        lib.ix_mlp_to_bf16.argtypes = [u64, vp, vp, vp]
        lib.ix_design_planes.argtypes = [vp, u32, vp, u32]
        lib.ix_design_planes.restype = u32
        lib.ix_design_material.argtypes = [vp, C.POINTER(abi.Material)]
        lib.ix_evaluate_designs.argtypes = [vp, vp, u32, C.POINTER(DesignView), vp]
        _bound = True
    return lib


def _ok(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("surrogate kernel launch failed")


# ---- designs and their traced metrics --------------------------------------------------
def sample_designs(n: int, seed: int) -> np.ndarray:
    """n designs uniform over the design box, [n, 12] float64."""
    rng = np.random.default_rng(seed)
    return LOWER + (UPPER - LOWER) * rng.random((n, N_FEATURES))


def normalize(designs: np.ndarray) -> np.ndarray:
    """The network's input: each parameter mapped from its range to [-1, 1]."""
    return ((designs - LOWER) / (UPPER - LOWER) * 2.0 - 1.0).astype(np.float32)


def _design_rows(designs: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(np.asarray(designs, np.float64).reshape(-1, N_FEATURES), np.float32)
    return d


def design_planes(design: np.ndarray, girdle_segments: int = 64) -> np.ndarray:
    """The design's f32 half-spaces [k, 4] (ix_design_planes)."""
    row = _design_rows(design)
    lib = _lib()
    k = lib.ix_design_planes(row.ctypes.data, girdle_segments, None, 0)
    if k == 0:
        raise ValueError("design out of its domain")
    out = np.zeros((k, 4), np.float32)
    lib.ix_design_planes(row.ctypes.data, girdle_segments, out.ctypes.data, k)
    return out


def design_material(design: np.ndarray) -> abi.Material:
    m = abi.Material()
    if _lib().ix_design_material(_design_rows(design).ctypes.data, C.byref(m)) != 0:
        raise ValueError("design out of its domain")
    return m


@dataclass
class RenderSpec:
    """How designs are traced: image size, samples per pixel, first sample, depth, the
    tilts (camera pitch from the table normal) and the girdle's segment count."""
    width: int = 32
    height: int = 32
    spp: int = 32
    sample_offset: int = 0
    max_bounces: int = 32
    girdle_segments: int = 64
    tilts_deg: Tuple[float, ...] = TILTS_DEG

    def paths_per_design(self) -> int:
        return self.width * self.height * self.spp * len(self.tilts_deg)


def _view(spec: RenderSpec):
    cams = (abi.Camera * len(spec.tilts_deg))()
    for i, t in enumerate(spec.tilts_deg):
        pitch = float(np.float32(math.pi / 2.0 - math.radians(t)))
        cams[i] = camera_new(0.0, pitch, FACE_UP_DISTANCE, FOV_DEG)
    env = environment_preset(PRESET_ISO_HEMISPHERE, 1.0, 0.0, 0.0, 0.0, 1.0, 20.0)
    view = DesignView(C.cast(cams, C.POINTER(abi.Camera)), len(spec.tilts_deg), spec.width, spec.height, spec.spp,
                      spec.sample_offset, spec.max_bounces, spec.girdle_segments, env)
    return view, cams


def evaluate_designs(backend: GpuBackend, designs: np.ndarray, spec: RenderSpec = RenderSpec(),
                     max_per_call: int = 4096) -> np.ndarray:
    """Traced metrics of every design, [n, 27]: brilliance at the 9 tilts, then fire, then
    scintillation (ix_evaluate_designs, one batched launch per `max_per_call` designs)."""
    if not backend.available:
        raise RuntimeError("no CUDA backend")
    rows = _design_rows(designs)
    n, t = rows.shape[0], len(spec.tilts_deg)
    out = np.zeros((n, t, 3), np.float32)
    view, cams = _view(spec)
    lib = _lib()
    for a in range(0, n, max_per_call):
        b = min(n, a + max_per_call)
        rc = lib.ix_evaluate_designs(backend._h, rows[a:].ctypes.data, b - a, C.byref(view),
                                     out[a:].ctypes.data)
        if rc != abi.IX_DONE:
            raise RuntimeError(f"design batch declined: {backend.last_lost_reason()}")
        global launches
        launches += int(backend.last_timing().launches)
    del cams
    return np.ascontiguousarray(out.transpose(0, 2, 1).reshape(n, N_OUTPUTS))


def tilt_means(metrics: np.ndarray) -> np.ndarray:
    """[n, 3]: each metric averaged over the tilts."""
    return metrics.reshape(metrics.shape[0], len(METRICS), -1).mean(axis=2)


def score(metrics: np.ndarray, scales: np.ndarray) -> np.ndarray:
    """A design's search score: the sum over the three metrics of its tilt-averaged value
    divided by that metric's scale (the training set's mean), so each counts alike."""
    return (tilt_means(metrics) / scales).sum(axis=1)


# ---- the network ----------------------------------------------------------------------
@dataclass
class Layer:
    w: object   # f32 [out, in] master weights (torch)
    wb: object  # bf16 copy
    b: object   # f32 [out]
    mw: object
    vw: object
    mb: object
    vb: object


class SurrogateMLP:
    """12 -> 256 -> 256 -> 256 -> 27 with SiLU between layers, MSE on standardised targets,
    Adam; BF16 GEMMs with FP32 accumulation on the tcgen05 kernels, FP32 master weights."""

    def __init__(self, dims: Sequence[int] = DIMS, seed: int = 0, device: str = "cuda") -> None:
        import torch

        self.torch = torch
        self.dev = torch.device(device)
        self.dims = tuple(int(d) for d in dims)
        g = np.random.default_rng(seed)
        self.layers: List[Layer] = []
        for fan_in, fan_out in zip(self.dims[:-1], self.dims[1:]):
            w = (g.standard_normal((fan_out, fan_in)) / math.sqrt(fan_in)).astype(np.float32)
            w = torch.from_numpy(w).to(self.dev)
            z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=self.dev)  # noqa: E731
            layer = Layer(w, torch.empty(fan_out, fan_in, dtype=torch.bfloat16, device=self.dev), z(fan_out),
                          z(fan_out, fan_in), z(fan_out, fan_in), z(fan_out), z(fan_out))
            _ok(_lib().ix_mlp_to_bf16(w.numel(), w.data_ptr(), layer.wb.data_ptr(), self._stream()))
            self.layers.append(layer)
        self.step = 0
        # Per-output standardisation of the targets (set by fit).
        self.t_mean = np.zeros(self.dims[-1], np.float32)
        self.t_std = np.ones(self.dims[-1], np.float32)

    def _stream(self) -> int:
        return self.torch.cuda.current_stream().cuda_stream

    def to_device_bf16(self, x: np.ndarray):
        global launches
        launches += 1
        torch = self.torch
        xt = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(self.dev)
        xb = torch.empty(xt.shape, dtype=torch.bfloat16, device=self.dev)
        _ok(_lib().ix_mlp_to_bf16(xt.numel(), xt.data_ptr(), xb.data_ptr(), self._stream()))
        return xb

    def forward_device(self, xb, keep: bool = False):
        """xb: bf16 [m, 12] on the device.  Returns the f32 output [m, 27] (standardised)
        and, with keep, per layer (bf16 input, f32 pre-activation)."""
        global launches
        torch, lib, s = self.torch, _lib(), self._stream()
        m = xb.shape[0]
        acts = []
        h = xb
        out = None
        launches += len(self.layers)
        for li, L in enumerate(self.layers):
            n, k = L.w.shape
            if li == len(self.layers) - 1:
                out = torch.empty(m, n, dtype=torch.float32, device=self.dev)
                _ok(lib.ix_mlp_linear(m, n, k, h.data_ptr(), k, L.wb.data_ptr(), L.b.data_ptr(), 0, None,
                                      out.data_ptr(), None, s))
                acts.append((h, None))
            else:
                z = torch.empty(m, n, dtype=torch.float32, device=self.dev) if keep else None
                hb = torch.empty(m, n, dtype=torch.bfloat16, device=self.dev)
                _ok(lib.ix_mlp_linear(m, n, k, h.data_ptr(), k, L.wb.data_ptr(), L.b.data_ptr(), 1,
                                      z.data_ptr() if keep else None, None, hb.data_ptr(), s))
                acts.append((h, z))
                h = hb
        return out, acts

    def predict(self, x: np.ndarray) -> np.ndarray:
        """Metrics [m, 27] of normalised designs x [m, 12]."""
        out, _ = self.forward_device(self.to_device_bf16(x))
        return out.cpu().numpy() * self.t_std + self.t_mean

    def gradients(self, x: np.ndarray, t: np.ndarray):
        """Loss and the f32 gradients [(dW [out, in], db)] of one batch (no update); t are
        the targets as the network sees them (standardised)."""
        return self._gradients_device(self.to_device_bf16(x),
                                      self.torch.from_numpy(np.ascontiguousarray(t, np.float32)).to(self.dev))

    def _gradients_device(self, xb, tt):
        torch, lib, s = self.torch, _lib(), self._stream()
        m = xb.shape[0]
        out, acts = self.forward_device(xb, keep=True)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        d_f32 = torch.empty_like(out)
        d_b16 = torch.empty(out.shape, dtype=torch.bfloat16, device=self.dev)
        _ok(lib.ix_mlp_mse_grad(m, out.shape[1], out.data_ptr(), tt.data_ptr(), d_f32.data_ptr(), d_b16.data_ptr(),
                                loss.data_ptr(), s))
        grads = [None] * len(self.layers)
        for li in range(len(self.layers) - 1, -1, -1):
            L = self.layers[li]
            h_in = acts[li][0]
            n, k = L.w.shape
            # dW = dZ^T h_in: (n x m) (m x k).
            dw = torch.empty(n, k, dtype=torch.float32, device=self.dev)
            _ok(lib.ix_mlp_gemm_bf16(1, 0, n, k, m, d_b16.data_ptr(), n, h_in.data_ptr(), k, dw.data_ptr(), k, s))
            db = torch.empty(n, dtype=torch.float32, device=self.dev)
            _ok(lib.ix_mlp_bias_grad(m, n, d_f32.data_ptr(), db.data_ptr(), s))
            grads[li] = (dw, db)
            if li > 0:
                # dZ_prev = (dZ W) * silu'(z_prev), fused in the GEMM's epilogue.
                z_prev = acts[li - 1][1]
                dz = torch.empty(m, k, dtype=torch.float32, device=self.dev)
                dzb = torch.empty(m, k, dtype=torch.bfloat16, device=self.dev)
                _ok(lib.ix_mlp_backward_silu(m, k, n, d_b16.data_ptr(), L.wb.data_ptr(), z_prev.data_ptr(),
                                             dz.data_ptr(), dzb.data_ptr(), s))
                d_f32, d_b16 = dz, dzb
        return loss, grads

    def _adam(self, grads, lr: float) -> None:
        lib, s = _lib(), self._stream()
        self.step += 1
        for L, (dw, db) in zip(self.layers, grads):
            _ok(lib.ix_mlp_adam(L.w.numel(), L.w.data_ptr(), L.wb.data_ptr(), dw.data_ptr(), L.mw.data_ptr(),
                                L.vw.data_ptr(), lr, 0.9, 0.999, 1e-8, self.step, s))
            _ok(lib.ix_mlp_adam(L.b.numel(), L.b.data_ptr(), None, db.data_ptr(), L.mb.data_ptr(), L.vb.data_ptr(),
                                lr, 0.9, 0.999, 1e-8, self.step, s))

    def train_step(self, x: np.ndarray, t: np.ndarray, lr: float = 1e-3) -> float:
        loss, grads = self.gradients(x, t)
        self._adam(grads, lr)
        return float(loss.item())

    def fit(self, x: np.ndarray, t: np.ndarray, epochs: int = 200, batch: int = 4096, lr: float = 1e-3,
            seed: int = 0, lr_final: Optional[float] = None) -> List[float]:
        """Adam on standardised targets; the data stays on the device and each epoch
        visits it in a fresh order.  lr decays geometrically to lr_final (default lr / 20)
        over the epochs.  Returns the mean loss of each epoch."""
        torch = self.torch
        self.t_mean = t.mean(axis=0).astype(np.float32)
        self.t_std = np.maximum(t.std(axis=0), 1e-6).astype(np.float32)
        ts = ((t - self.t_mean) / self.t_std).astype(np.float32)
        xb_all = self.to_device_bf16(x)
        t_all = torch.from_numpy(ts).to(self.dev)
        n = x.shape[0]
        g = torch.Generator(device="cpu")
        g.manual_seed(seed)
        lr_final = lr / 20.0 if lr_final is None else lr_final
        decay = (lr_final / lr) ** (1.0 / max(1, epochs - 1))
        losses = []
        for ep in range(epochs):
            order = torch.randperm(n, generator=g).to(self.dev)
            total = torch.zeros((), dtype=torch.float32, device=self.dev)
            steps = 0
            for i in range(0, n, batch):
                idx = order[i:i + batch]
                loss, grads = self._gradients_device(xb_all[idx].contiguous(), t_all[idx].contiguous())
                self._adam(grads, lr * decay ** ep)
                total += loss[0]
                steps += 1
            losses.append(float(total.item()) / steps)
        return losses

    def refine(self, x: np.ndarray, t: np.ndarray, steps: int = 10, batch: int = 256, lr: float = 2e-4,
               seed: int = 0) -> None:
        """A few Adam steps on (x, t) under the standardisation fit() set, the moments
        carried on: a search feeds it the designs it has traced, so the network sharpens
        where the search is going."""
        torch = self.torch
        ts = ((t - self.t_mean) / self.t_std).astype(np.float32)
        xb_all = self.to_device_bf16(x)
        t_all = torch.from_numpy(ts).to(self.dev)
        n = x.shape[0]
        rng = np.random.default_rng(seed)
        for _ in range(steps):
            idx = torch.from_numpy(rng.integers(0, n, min(batch, n))).to(self.dev)
            _, grads = self._gradients_device(xb_all[idx].contiguous(), t_all[idx].contiguous())
            self._adam(grads, lr)


class SurrogateEnsemble:
    """`members` networks of the same shape from different seeds, trained on the same data
    in different orders; the spread of their scores is the disagreement."""

    def __init__(self, members: int = 4, seed: int = 0, dims: Sequence[int] = DIMS) -> None:
        self.nets = [SurrogateMLP(dims, seed=seed + 1000 * i) for i in range(members)]

    def fit(self, x: np.ndarray, t: np.ndarray, **kw) -> List[List[float]]:
        seed = kw.pop("seed", 0)
        return [net.fit(x, t, seed=seed + i, **kw) for i, net in enumerate(self.nets)]

    def refine(self, x: np.ndarray, t: np.ndarray, steps: int = 10, seed: int = 0) -> None:
        for i, net in enumerate(self.nets):
            net.refine(x, t, steps=steps, seed=seed + i)

    def predict_members(self, x: np.ndarray) -> np.ndarray:
        """[members, m, 27]; one bf16 upload shared by all members."""
        xb = self.nets[0].to_device_bf16(x)
        outs = [net.forward_device(xb)[0] for net in self.nets]
        return np.stack([o.cpu().numpy() * net.t_std + net.t_mean for o, net in zip(outs, self.nets)])

    def predict(self, x: np.ndarray) -> np.ndarray:
        return self.predict_members(x).mean(axis=0)

    def score(self, x: np.ndarray, scales: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(mean metrics [m, 27], mean score [m], disagreement [m]): the members' score
        standard deviation relative to their mean score."""
        pm = self.predict_members(x)
        per = np.stack([score(p, scales) for p in pm])
        mean = per.mean(axis=0)
        return pm.mean(axis=0), mean, per.std(axis=0) / np.maximum(np.abs(mean), 1e-12)


# ---- design search --------------------------------------------------------------------
@dataclass
class SearchConfig:
    population: int = 4096
    generations: int = 50
    elite: int = 64          # designs per generation the tracer re-renders / keeps
    sigma: float = 0.05      # mutation step, fraction of each parameter's range
    fallback: float = 0.02   # ensemble disagreement above which the tracer scores a design
    refine_steps: int = 10   # screened search: Adam steps per member on the traced designs, per generation
    seed: int = 0


@dataclass
class SearchResult:
    best_design: np.ndarray
    best_metrics: np.ndarray       # traced at the search's fidelity
    best_score: float
    history: List[float] = field(default_factory=list)  # best traced score after each generation
    evaluations: int = 0           # candidates scored (by the network or the tracer)
    traced: int = 0                # designs the tracer rendered
    fallbacks: int = 0             # candidates the tracer scored because the ensemble disagreed
    seconds: float = 0.0           # wall time of the generations, device work synchronised

    @property
    def evals_per_s(self) -> float:
        return self.evaluations / self.seconds if self.seconds > 0 else 0.0


def _offspring(rng: np.random.Generator, parents: np.ndarray, n: int, sigma: float,
               keep_parents: bool = True) -> np.ndarray:
    """n children of the parents: uniform crossover of two random parents, a Gaussian step
    of sigma x range per parameter, clipped to the box; with keep_parents the parents
    come first."""
    k = parents.shape[0]
    a = parents[rng.integers(0, k, n)]
    b = parents[rng.integers(0, k, n)]
    mask = rng.random(a.shape) < 0.5
    child = np.where(mask, a, b) + rng.standard_normal(a.shape) * sigma * (UPPER - LOWER)
    child = np.clip(child, LOWER, UPPER)
    if keep_parents:
        child[:min(k, n)] = parents[:min(k, n)]
    return child


def _next_elite(elite_d, elite_m, new_d, new_m, scales, k):
    """The best k of the current elite and the newly traced designs, by traced score."""
    if elite_d is not None:
        new_d = np.concatenate([elite_d, new_d])
        new_m = np.concatenate([elite_m, new_m])
    order = np.argsort(-score(new_m, scales), kind="stable")[:k]
    return new_d[order], new_m[order]


def traced_search(backend: GpuBackend, scales: np.ndarray, cfg: SearchConfig = SearchConfig(),
                  spec: RenderSpec = RenderSpec(), evaluate=None) -> SearchResult:
    """Evolutionary search in which the tracer scores every candidate: each generation
    traces `population` children of the elite, and the elite becomes the best cfg.elite
    of itself and the children by traced score.  `evaluate` (designs -> metrics [n, 27])
    defaults to evaluate_designs on `backend` with `spec`."""
    if evaluate is None:
        evaluate = lambda d: evaluate_designs(backend, d, spec)  # noqa: E731
    rng = np.random.default_rng(cfg.seed)
    pop = sample_designs(cfg.population, cfg.seed)
    elite_d = elite_m = None
    res = SearchResult(np.zeros(N_FEATURES), np.zeros(N_OUTPUTS), -np.inf)
    t0 = time.perf_counter()
    for _ in range(cfg.generations):
        m = evaluate(pop)
        elite_d, elite_m = _next_elite(elite_d, elite_m, pop, m, scales, cfg.elite)
        res.evaluations += len(pop)
        res.traced += len(pop)
        res.history.append(float(score(elite_m[:1], scales)[0]))
        pop = _offspring(rng, elite_d, cfg.population, cfg.sigma, keep_parents=False)
    res.seconds = time.perf_counter() - t0
    res.best_design, res.best_metrics, res.best_score = elite_d[0].copy(), elite_m[0].copy(), res.history[-1]
    return res


def screened_search(backend: GpuBackend, ensemble: SurrogateEnsemble, scales: np.ndarray,
                    cfg: SearchConfig = SearchConfig(), spec: RenderSpec = RenderSpec(),
                    evaluate=None) -> SearchResult:
    """Evolutionary search in which the ensemble scores every candidate.  Each generation
    scores `population` children of the elite with the ensemble; children whose ensemble
    disagreement exceeds cfg.fallback are scored by the tracer instead, the best
    cfg.elite children by that score are rendered by the tracer, and the elite becomes the
    best cfg.elite of itself and every traced child by traced score -- so every reported
    metric is a traced one and the elite never gets worse.  After each generation every
    member takes cfg.refine_steps Adam steps on all the designs this search has traced
    (the tracer's renders are the surrogate's training data: where the search goes, the
    network sharpens).  `evaluate` as for traced_search."""
    if evaluate is None:
        evaluate = lambda d: evaluate_designs(backend, d, spec)  # noqa: E731
    rng = np.random.default_rng(cfg.seed)
    pop = sample_designs(cfg.population, cfg.seed)
    elite_d = elite_m = None
    seen_d, seen_m = [], []
    res = SearchResult(np.zeros(N_FEATURES), np.zeros(N_OUTPUTS), -np.inf)
    t0 = time.perf_counter()
    for _ in range(cfg.generations):
        _, s, dis = ensemble.score(normalize(pop), scales)
        fb = np.flatnonzero(dis > cfg.fallback)
        traced = {}
        if fb.size:
            m_fb = evaluate(pop[fb])
            s[fb] = score(m_fb, scales)
            traced.update({int(i): m_fb[j] for j, i in enumerate(fb)})
        top = np.argsort(-s, kind="stable")[:cfg.elite]
        redo = np.array([i for i in top if int(i) not in traced], np.int64)
        if redo.size:
            m_re = evaluate(pop[redo])
            traced.update({int(i): m_re[j] for j, i in enumerate(redo)})
        idx = np.array(sorted(traced), np.int64)
        new_m = np.stack([traced[int(i)] for i in idx])
        elite_d, elite_m = _next_elite(elite_d, elite_m, pop[idx], new_m, scales, cfg.elite)
        if cfg.refine_steps > 0 and hasattr(ensemble, "refine"):
            seen_d.append(pop[idx])
            seen_m.append(new_m)
            ensemble.refine(normalize(np.concatenate(seen_d)), np.concatenate(seen_m), steps=cfg.refine_steps,
                            seed=cfg.seed + len(seen_d))
        res.evaluations += len(pop)
        res.traced += fb.size + redo.size
        res.fallbacks += fb.size
        res.history.append(float(score(elite_m[:1], scales)[0]))
        pop = _offspring(rng, elite_d, cfg.population, cfg.sigma, keep_parents=False)
    res.seconds = time.perf_counter() - t0
    res.best_design, res.best_metrics, res.best_score = elite_d[0].copy(), elite_m[0].copy(), res.history[-1]
    return res


def relative_error(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """|a - b| / |b| per tilt-averaged metric ([3]) of one design's metrics [27]."""
    ta, tb = tilt_means(a.reshape(1, -1))[0], tilt_means(b.reshape(1, -1))[0]
    return np.abs(ta - tb) / np.maximum(np.abs(tb), 1e-12)
