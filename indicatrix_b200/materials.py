"""Material PODs (``ix_material``) for the built-in and generated gem materials.

Each builder fills the fields the transport reads from the reference's ``GemMaterial``
(crates/indicatrix/src/optics/materials/mod.rs:116-236).
"""
from __future__ import annotations

import numpy as np

from . import abi


def _base(dispersion: abi.Dispersion) -> abi.Material:
    m = abi.Material()
    m.dispersion = dispersion
    m.anisotropic = 0
    m.birefringence_delta = 0.0
    m.c_axis[:] = [0.0, 1.0, 0.0]
    m.absorption_path_scale = 1.0
    m.edge_rounding_radius = 0.0
    m.scattering_sigma_s = 0.0
    return m


def sellmeier3(b, c) -> abi.Dispersion:
    d = abi.Dispersion()
    d.kind = abi.DISP_SELLMEIER3
    d.b[:] = [float(x) for x in b]
    d.c[:] = [float(x) for x in c]
    return d


def cauchy(a: float, b: float, c: float = 0.0) -> abi.Dispersion:
    d = abi.Dispersion()
    d.kind = abi.DISP_CAUCHY
    d.b[:] = [float(a), float(b), float(c)]
    d.c[:] = [0.0, 0.0, 0.0]
    return d


def diamond() -> abi.Material:
    """Diamond: Peter (1923) two-term Sellmeier with the third pole zeroed, colourless
    (materials/diamond_through_emerald.rs:29-57)."""
    return _base(sellmeier3([4.3356, 0.3306, 0.0], [0.011236, 0.030625, 1.0]))


def isotropic(dispersion: abi.Dispersion, spline_alpha=None, path_scale: float = 1.0) -> abi.Material:
    """A cubic (isotropic) material with an optional tabulated absorption spline
    (IX_SPLINE_KNOTS values of alpha in 1/length over 380-780 nm)."""
    m = _base(dispersion)
    if spline_alpha is not None:
        knots = np.asarray(spline_alpha, np.float32)
        assert knots.shape == (abi.SPLINE_KNOTS,)
        for ab in (m.abs_o, m.abs_e):
            ab.has_spline = 1
            ab.spline[:] = [float(x) for x in knots]
    m.absorption_path_scale = float(path_scale)
    return m
