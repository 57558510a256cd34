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
    m.scattering_g = 0.0
    return m


def with_scattering(m: abi.Material, sigma_s: float, g: float) -> abi.Material:
    """GemMaterial::with_scattering: Henyey-Greenstein interior scattering, sigma_s per
    model unit and asymmetry g (optics/materials/mod.rs)."""
    m.scattering_sigma_s = float(sigma_s)
    m.scattering_g = float(g)
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


def energy_band(center_nm: float, fwhm_cm_inv: float, peak: float) -> abi.Band:
    """AbsorptionBand::energy (optics/absorption.rs:95): a Gaussian in wavenumber whose
    width field holds sigma = FWHM / 2.35482, rounded in f32."""
    b = abi.Band()
    b.center_nm = float(center_nm)
    b.width_nm = float(np.float32(fwhm_cm_inv) / np.float32(2.35482))
    b.peak = float(peak)
    b.shape = abi.BAND_GAUSS_ENERGY
    return b


def _set_bands(ab: abi.Absorption, bands) -> None:
    assert len(bands) <= abi.MAX_BANDS
    ab.n_bands = len(bands)
    for i, b in enumerate(bands):
        ab.bands[i] = b


def uniaxial(dispersion: abi.Dispersion, delta: float, c_axis=(0.0, 1.0, 0.0), o_bands=(), e_bands=(),
             e_dispersion: abi.Dispersion | None = None) -> abi.Material:
    """A uniaxial material (GemMaterial with crystal_system != Cubic and
    |birefringence_delta| > 1e-4, transport/inner.rs:183): ordinary dispersion, the
    constant-offset or separate extraordinary index, the optic axis as stored, and the
    o-ray / e-ray absorption bands."""
    m = _base(dispersion)
    m.anisotropic = 1 if abs(float(np.float32(delta))) > 1e-4 else 0
    m.birefringence_delta = float(delta)
    m.c_axis[:] = [float(x) for x in c_axis]
    if e_dispersion is not None:
        m.has_e_dispersion = 1
        m.e_dispersion = e_dispersion
    _set_bands(m.abs_o, list(o_bands))
    _set_bands(m.abs_e, list(e_bands))
    return m


def sapphire(c_axis=(0.0, 1.0, 0.0)) -> abi.Material:
    """Sapphire (materials/diamond_through_emerald.rs:74-140): Malitson-o three-term
    Sellmeier, birefringence -0.0081, optic axis +Y, Fe-Ti pleochroic o/e energy bands."""
    return uniaxial(
        sellmeier3([1.431349, 0.650547, 5.341402], [0.00528, 0.01424, 325.015]), -0.0081, c_axis,
        o_bands=[energy_band(585.0, 4878.0, 2.01), energy_band(744.0, 3142.0, 0.887),
                 energy_band(457.0, 12000.0, 0.433)],
        e_bands=[energy_band(612.0, 7466.0, 0.371), energy_band(729.0, 4955.0, 1.03),
                 energy_band(467.0, 11169.0, 0.524)])


def wavelength_band(center_nm: float, width_nm: float, peak: float) -> abi.Band:
    """AbsorptionBand::new (optics/absorption.rs): a Gaussian in wavelength."""
    b = abi.Band()
    b.center_nm, b.width_nm, b.peak = float(center_nm), float(width_nm), float(peak)
    b.shape = abi.BAND_GAUSS_WAVELENGTH
    return b


def quartz(c_axis=(0.0, 1.0, 0.0)) -> abi.Material:
    """Quartz (materials/spinel_through_tourmaline.rs:76-118): Ghosh o-ray Sellmeier and
    its own e-ray Sellmeier (a separate extraordinary dispersion curve), colourless."""
    return uniaxial(sellmeier3([0.2860414, 1.0704408, 1.1020224], [0.0, 0.0100586, 100.0]), 0.0091, c_axis,
                    e_dispersion=sellmeier3([0.28851804, 1.0950992, 1.1566248], [0.0, 0.010210186, 100.0]))


def rutile(c_axis=(0.0, 1.0, 0.0)) -> abi.Material:
    """Rutile (materials/rutile.rs:54-80): extreme positive birefringence (0.2957) with
    o- and e-ray Sellmeier fits and a UV band on both rays."""
    band = [wavelength_band(350.0, 40.0, 8.0)]
    return uniaxial(sellmeier3([3.039851, 1.873149, 0.0], [0.0803, 0.0, 0.0]), 0.2957, c_axis,
                    o_bands=band, e_bands=band,
                    e_dispersion=sellmeier3([3.940688, 2.256312, 0.0], [0.0843, 0.0, 0.0]))
