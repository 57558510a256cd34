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


def biaxial(dispersion: abi.Dispersion, delta: float, delta_beta_alpha: float, c_axis=(0.0, 1.0, 0.0),
            alpha_bands=(), beta_bands=None, gamma_bands=()) -> abi.Material:
    """A biaxial material (GemMaterial with biaxial_delta_beta_alpha set,
    materials/optics.rs:16): n_beta from the dispersion, n_alpha = n_beta - delta_beta_alpha,
    n_gamma = n_alpha + delta, gamma axis along c_axis; alpha / beta / gamma ray absorption
    (AbsorptionTensor::biaxial, optics/absorption.rs:338).  Without beta bands the beta axis
    absorbs as the alpha ray (AbsorptionTensor::isotropic / uniaxial carry no beta_ray)."""
    m = uniaxial(dispersion, delta, c_axis, o_bands=alpha_bands, e_bands=gamma_bands)
    m.biaxial = 1
    m.biaxial_delta_beta_alpha = float(delta_beta_alpha)
    if beta_bands is not None:
        m.has_abs_beta = 1
        _set_bands(m.abs_beta, list(beta_bands))
    return m


def alexandrite(c_axis=(0.0, 1.0, 0.0)) -> abi.Material:
    """Alexandrite (materials/zircon_through_topaz.rs:108-195): three-term Sellmeier,
    birefringence 0.0076, n_beta - n_alpha 0.001951, trichroic Cr3+ wavelength bands."""
    w = wavelength_band
    return biaxial(sellmeier3([0.78522, 1.21202, 16.81], [0.0, 0.01262, 1000.0]), 0.0076, 0.001951, c_axis,
                   alpha_bands=[w(565.0, 40.0, 1.9), w(420.0, 32.0, 1.8)],
                   beta_bands=[w(560.0, 40.0, 0.65), w(422.0, 32.0, 3.5)],
                   gamma_bands=[w(595.0, 40.0, 3.1), w(430.0, 32.0, 1.5)])


def topaz(c_axis=(0.0, 1.0, 0.0)) -> abi.Material:
    """Topaz (materials/zircon_through_topaz.rs:230-257): Cauchy, birefringence 0.008,
    n_beta - n_alpha 0.0024, one isotropic wavelength band (no beta ray)."""
    band = [wavelength_band(620.0, 70.0, 1.6)]
    return biaxial(cauchy(1.614872, 0.004273), 0.0080, 0.0024, c_axis, alpha_bands=band, gamma_bands=band)


def tanzanite(c_axis=(0.0, 1.0, 0.0)) -> abi.Material:
    """Tanzanite (materials/tanzanite_through_cubic_zirconia.rs:13-40, :66-160): Cauchy,
    birefringence 0.013, n_beta - n_alpha 0.0025, trichroic V3+ energy bands."""
    e = energy_band
    return biaxial(cauchy(1.674589, 0.009123), 0.0130, 0.0025, c_axis,
                   alpha_bands=[e(350.0, 5083.0, 4.81), e(505.0, 5500.0, 2.11), e(577.0, 3037.0, 2.36),
                                e(751.0, 2191.0, 0.326)],
                   beta_bands=[e(340.0, 5683.0, 12.2), e(565.0, 5493.0, 2.1), e(610.0, 1526.0, 0.873),
                               e(771.0, 2423.0, 2.26)],
                   gamma_bands=[e(385.0, 2560.0, 9.86), e(440.0, 3095.0, 0.508), e(538.0, 3664.0, 1.35),
                                e(612.0, 2209.0, 1.73), e(742.0, 2551.0, 1.33)])


def peridot(c_axis=(0.0, 1.0, 0.0)) -> abi.Material:
    """Peridot (materials/peridot_through_benitoite.rs:13-95): Cauchy, birefringence 0.036,
    n_beta - n_alpha 0.015, trichroic Fe2+ energy bands."""
    e = energy_band
    return biaxial(cauchy(1.636549, 0.006062), 0.036, 0.0150, c_axis,
                   alpha_bands=[e(345.0, 10096.0, 5.38), e(455.0, 1410.0, 0.53), e(490.0, 2160.0, 0.44),
                                e(637.0, 1724.0, 0.80), e(840.0, 3276.0, 4.76), e(1000.0, 2534.0, 35.2)],
                   beta_bands=[e(341.0, 12000.0, 6.78), e(465.0, 2526.0, 1.07), e(500.0, 3000.0, 0.47),
                               e(635.0, 2500.0, 1.33), e(840.0, 4000.0, 4.25), e(1000.0, 2401.0, 35.2)],
                   gamma_bands=[e(376.0, 3317.0, 4.77), e(440.0, 2933.0, 2.24), e(500.0, 3000.0, 0.79),
                                e(627.0, 2500.0, 0.77), e(840.0, 4000.0, 2.34), e(1000.0, 3663.0, 12.7)])
