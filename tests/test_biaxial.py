"""The oracle's biaxial indicatrix against the reference's own biaxial tests.

The reference holds no golden vectors for the biaxial transport; its known-answer and
property tests (crates/indicatrix/src/optics/birefringence/tests/biaxial_reduction.rs)
pin the indicatrix, and they are restated here against the oracle's functions (through
``ixo_biaxial_bundle``), with the reference's tolerances.  The transport built on it is
then checked end to end: a lossless biaxial stone keeps the
white furnace, and biaxial renders differ measurably from the uniaxial approximation, as
the reference's wiring tests ask
(tests/raytracer_tests/pleochroic_biaxial_wiring.rs).
"""
import ctypes as C
import math

import numpy as np
import pytest

from indicatrix_b200 import abi, materials

pytestmark = pytest.mark.filterwarnings("ignore::RuntimeWarning")


@pytest.fixture(scope="module")
def oracle():
    from oracle import ix_oracle
    return ix_oracle


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def bundle(oracle, m: abi.Material, k, normal=(0.0, 1.0, 0.0), cos_i=0.8, lam=589.3) -> np.ndarray:
    k = np.ascontiguousarray(k, np.float32)
    n = np.ascontiguousarray(normal, np.float32)
    out = np.zeros(24, np.float32)
    n_beta = oracle.lib().ixo_dispersion_eval(C.byref(m.dispersion), C.c_float(lam))
    oracle.lib().ixo_biaxial_bundle(C.byref(m), _p(k), _p(n), C.c_float(cos_i), C.c_float(lam), C.c_float(n_beta),
                                    _p(out))
    return out


def constant_index(n: float) -> abi.Dispersion:
    return materials.cauchy(n, 0.0, 0.0)


def unit(v) -> np.ndarray:
    v = np.asarray(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


def stable_basis(nv):
    """stable_orthonormal_basis (birefringence/helpers.rs:13) in f32."""
    nv = np.asarray(nv, np.float32)
    a = np.array([0, 1, 0], np.float32) if abs(nv[0]) > 0.9 else np.array([1, 0, 0], np.float32)
    t = a - nv * np.float32(np.dot(nv, a))
    t = t / np.float32(np.sqrt(np.dot(t, t)))
    return t, np.cross(nv, t).astype(np.float32)


def effective_e_index(n_o, n_e, theta):
    """effective_extraordinary_index (birefringence/uniaxial.rs:33) in f64."""
    s, c = math.sin(theta), math.cos(theta)
    return n_o * n_e / math.sqrt((n_e * c) ** 2 + (n_o * s) ** 2)


def test_wave_indices_reduce_to_the_uniaxial_formula(oracle):
    """biaxial_reduction.rs:21: n_alpha == n_beta is the uniaxial closed form, 1e-3."""
    n_o, n_e = 1.65, 1.72
    c_axis = unit([0.35, 0.82, -0.45])
    m = materials.biaxial(constant_index(n_o), n_e - n_o, 0.0, c_axis)
    for d in ([1, 0, 0], [0, 1, 0], [0, 0, 1], c_axis, [0.2, 0.9, 0.1], [-0.5, 0.3, 0.8], [0.7, -0.6, 0.2],
              [0.1, 0.1, 0.99], [-0.9, -0.3, 0.2]):
        w = unit(d)
        out = bundle(oracle, m, w)
        theta = math.acos(min(1.0, abs(float(np.dot(w, c_axis)))))
        n_eff = effective_e_index(n_o, n_e, theta)
        assert abs(out[1] - min(n_o, n_eff)) < 1e-3
        assert abs(out[0] - max(n_o, n_eff)) < 1e-3


def test_wave_indices_reduce_to_isotropic_when_all_equal(oracle):
    """biaxial_reduction.rs:63."""
    m = materials.biaxial(constant_index(1.9), 0.0, 0.0)
    for d in ([1, 0, 0], [0, 1, 0], [0, 0, 1], [0.3, 0.5, 0.8]):
        out = bundle(oracle, m, unit(d))
        assert abs(out[0] - 1.9) < 1e-4 and abs(out[1] - 1.9) < 1e-4


def test_eigen_polarizations_are_orthonormal_and_transverse(oracle):
    """biaxial_reduction.rs:90 (indices 1.60 / 1.65 / 1.75)."""
    m = materials.biaxial(constant_index(1.65), 0.15, 0.05, (0.0, 0.0, 1.0))
    for d in ([0.3, 0.5, 0.8], [0.9, 0.1, -0.2], [-0.4, 0.6, 0.5]):
        w = unit(d)
        out = bundle(oracle, m, w)
        ds, df = out[2:5], out[5:8]
        assert np.all(np.isfinite(out[:8]))
        assert abs(np.linalg.norm(ds) - 1) < 1e-3 and abs(np.linalg.norm(df) - 1) < 1e-3
        assert abs(np.dot(ds, df)) < 1e-2
        assert abs(np.dot(ds, w)) < 1e-2 and abs(np.dot(df, w)) < 1e-2


@pytest.mark.parametrize("name", ["alexandrite", "topaz", "tanzanite"])
def test_eigenvectors_satisfy_the_eigen_equation_across_a_dense_sweep(oracle, name):
    """biaxial_reduction.rs:150: D_i (x - b_i) = -k_i (k . E), E_j = b_j D_j, residual
    < 2e-4 over a 181-sample great-circle arc at 589.3 nm, unit length, and the eigen
    line continuous (|dot| > 0.98 between neighbours)."""
    m = getattr(materials, name)()
    n_beta = np.float32(oracle.lib().ixo_dispersion_eval(C.byref(m.dispersion), C.c_float(589.3)))
    na = np.float32(n_beta - np.float32(m.biaxial_delta_beta_alpha))
    ng = np.float32(na + np.float32(m.birefringence_delta))
    b = np.array([1 / (float(na) ** 2), 1 / (float(n_beta) ** 2), 1 / (float(ng) ** 2)])
    g = unit(m.c_axis[:])
    a1, a2 = stable_basis(g)
    axes = np.stack([a1, a2, g], axis=1).astype(np.float64)
    u, v = unit([0.4, 0.6, 0.69]), unit([0.8, -0.3, 0.2])
    prev = [None, None]
    for i in range(181):
        th = np.float32(i) / np.float32(180.0) * np.float32(math.pi)
        k = unit(np.float32(math.cos(th)) * u + np.float32(math.sin(th)) * v)
        out = bundle(oracle, m, k)
        local = axes.T @ k.astype(np.float64)
        for j, (n, d) in enumerate(((out[0], out[2:5]), (out[1], out[5:8]))):
            assert abs(np.linalg.norm(d) - 1) < 1e-4
            x = 1.0 / (float(n) ** 2)
            dl = axes.T @ d.astype(np.float64)
            e_dot_k = float(np.dot(local * b, dl))
            residual = dl * (x - b) + local * e_dot_k
            assert np.linalg.norm(residual) < 2e-4, (name, i, j)
            if prev[j] is not None:
                assert abs(float(np.dot(prev[j], d))) > 0.98, (name, i, j)
            prev[j] = d


def test_discriminant_reformulation_matches_the_naive_form():
    """biaxial_reduction.rs:233: precise_root_near's discriminant equals B^2 - 4C (f64)."""
    rng = np.random.default_rng(7)
    for _ in range(200):
        k = rng.normal(size=3)
        k /= np.linalg.norm(k)
        a, bb, cc = k * k
        p, q, r = 1 / rng.uniform(1.4, 2.6, size=3) ** 2
        big_b = a * (q + r) + bb * (p + r) + cc * (p + q)
        big_c = a * q * r + bb * p * r + cc * p * q
        naive = big_b * big_b - 4 * big_c
        x, y = p - q, r - p
        reform = (a + cc) ** 2 * x * x + 2 * (a - bb * cc) * x * y + (a + bb) ** 2 * y * y
        assert abs(naive - reform) <= 1e-12 * max(1.0, abs(naive))


def test_mode_poynting_dir_is_a_unit_vector_perpendicular_to_its_field(oracle):
    """biaxial_reduction.rs:301-330 through mode_poynting_dir: S is unit, finite and
    perpendicular to the mode's E (E = eps^-1 D); S leans towards k (S . k > 0)."""
    m = materials.tanzanite()
    rng = np.random.default_rng(3)
    n_beta = float(np.float32(oracle.lib().ixo_dispersion_eval(C.byref(m.dispersion), C.c_float(589.3))))
    n = np.array([n_beta - m.biaxial_delta_beta_alpha, n_beta,
                  n_beta - m.biaxial_delta_beta_alpha + m.birefringence_delta])
    g = unit(m.c_axis[:])
    a1, a2 = stable_basis(g)
    axes = np.stack([a1, a2, g], axis=1).astype(np.float64)
    for _ in range(64):
        k = unit(rng.normal(size=3))
        out = bundle(oracle, m, k)
        for d, s in ((out[2:5], out[8:11]), (out[5:8], out[11:14])):
            e = axes @ ((axes.T @ d.astype(np.float64)) / n ** 2)
            e /= np.linalg.norm(e)
            assert np.all(np.isfinite(s)) and abs(np.linalg.norm(s) - 1) < 1e-4
            assert abs(float(np.dot(s, e))) < 1e-3
            assert float(np.dot(s, k)) > 0.99


def test_resolve_entry_mode_obeys_snell_law_at_its_own_index(oracle):
    """resolve_entry_mode (biaxial.rs:370): after two fixed-point steps the returned
    wave normal refracts at the returned index to within the fixed point's residual, and
    the two modes' indices straddle n_beta."""
    m = materials.peridot()
    rng = np.random.default_rng(11)
    normal = np.array([0.0, 1.0, 0.0], np.float32)
    for _ in range(64):
        cos_i = float(rng.uniform(0.2, 1.0))
        sin_i = math.sqrt(1 - cos_i * cos_i)
        phi = rng.uniform(0, 2 * math.pi)
        k = np.array([sin_i * math.cos(phi), -cos_i, sin_i * math.sin(phi)], np.float32)
        out = bundle(oracle, m, k, normal, cos_i)
        for n, d in ((out[14], out[15:18]), (out[18], out[19:22])):
            sin_t = math.sqrt(max(0.0, 1 - float(np.dot(d, -normal)) ** 2))
            assert abs(sin_t * n - sin_i) < 2e-3, (n, sin_t, sin_i)
        assert out[14] >= out[18]


def test_absorption_frame_worked_example_and_principal_coefficients(oracle):
    """biaxial_reduction.rs:384 and :407: with the gamma axis +Y the alpha axis is +X and
    the beta axis -Z, so the biaxial tensor's quadratic form returns alpha / beta / gamma
    for a field along X / Z / Y; with the beta ray equal to the alpha ray the form is the
    uniaxial one (:438)."""
    a1, a2 = stable_basis(np.array([0, 1, 0], np.float32))
    assert np.allclose(a1, [1, 0, 0]) and np.allclose(a2, [0, 0, -1])
    # A material absorbing 1.5 / 4 / 9 per unit on the alpha / beta / gamma rays at all
    # wavelengths, probed through the assigned-mode alpha of a wave normal whose mode
    # fields lie on the principal axes: k along the gamma axis (+Y) has its two modes on
    # alpha (+X) and beta (-Z).
    w = materials.wavelength_band
    flat = lambda peak: [w(580.0, 1e6, peak)]
    m = materials.biaxial(constant_index(1.6), 0.15, 0.05, (0.0, 1.0, 0.0), alpha_bands=flat(1.5),
                          beta_bands=flat(4.0), gamma_bands=flat(9.0))
    out = bundle(oracle, m, np.array([0, 1, 0], np.float32))
    assert sorted([round(float(out[22]), 3), round(float(out[23]), 3)]) == [1.5, 4.0]
    out = bundle(oracle, m, np.array([1, 0, 0], np.float32))
    assert sorted([round(float(out[22]), 3), round(float(out[23]), 3)]) == [4.0, 9.0]
    m_u = materials.biaxial(constant_index(1.6), 0.15, 0.05, (0.0, 1.0, 0.0), alpha_bands=flat(1.5),
                            beta_bands=flat(1.5), gamma_bands=flat(9.0))
    m_n = materials.biaxial(constant_index(1.6), 0.15, 0.05, (0.0, 1.0, 0.0), alpha_bands=flat(1.5),
                            gamma_bands=flat(9.0))
    for d in ([0.4, -0.5, 0.77], [0.2, 0.6, 0.77], [1, 0, 0]):
        a = bundle(oracle, m_u, unit(d))
        b = bundle(oracle, m_n, unit(d))
        assert a[22:24].tobytes() == b[22:24].tobytes()


def _scene(oracle, material, width=24, height=24, max_bounces=24, preset=1):
    planes = np.ascontiguousarray(oracle.standard_round_brilliant())
    sc = abi.Scene()
    sc.camera = oracle.camera_new(0.0, 0.5, 6.0, 30.0)
    sc.width, sc.height = width, height
    sc.planes = _p(planes)
    sc.n_planes = planes.shape[0]
    sc.material = material
    sc.max_bounces = max_bounces
    sc.environment = oracle.environment_preset(preset, 1.0, 0.3, 0.8)
    return sc, planes


def test_biaxial_white_furnace(oracle):
    """A colourless, non-dispersive biaxial stone (n_beta 1.5, n_alpha 1.49, n_gamma 1.52)
    in a uniform environment returns the environment's radiance within the 0.025 of the
    reference's furnace anchors (white_furnace_energy_conservation.rs), 96 samples per
    pixel of the 12 x 12 furnace grid, depth 12."""
    from test_frosted import furnace_scene, furnace_target

    mat = materials.biaxial(constant_index(1.5), 0.03, 0.01)
    sc, _keep = furnace_scene(oracle, mat, finishes=False)
    _, s64, dropped = oracle.trace_frame(sc, 0, 96, threads=0)
    assert dropped == 0
    mean = s64.reshape(-1, 3).sum(axis=0) / (12 * 12 * 96)
    target = furnace_target(oracle)
    assert np.all(np.abs(mean - target) / target <= 0.025), (mean, target)


@pytest.mark.parametrize("name", ["alexandrite", "topaz", "tanzanite", "peridot"])
def test_biaxial_renders_are_finite_and_differ_from_the_uniaxial_approximation(oracle, name):
    """pleochroic_biaxial_wiring.rs:28 and :288: every biaxial built-in renders finite,
    non-negative XYZ, and the biaxial transport differs measurably from the same material
    traced as uniaxial (biaxial flag off)."""
    m = getattr(materials, name)()
    sc, planes = _scene(oracle, m)
    _, xyz, _ = oracle.trace_frame(sc, 0, 32, threads=0)
    assert np.all(np.isfinite(xyz)) and np.all(xyz >= 0) and xyz[..., 1].sum() > 0
    mu = getattr(materials, name)()
    mu.biaxial = 0
    su, pu = _scene(oracle, mu)
    _, xu, _ = oracle.trace_frame(su, 0, 32, threads=0)
    rel = np.abs(xyz - xu).sum() / xu.sum()
    assert rel > 1e-3, rel


def test_biaxial_routing():
    """The routing predicate (host code of the C ABI, no GPU needed): a biaxial material
    routes to the GPU; a biaxial indicatrix on a material not marked anisotropic is
    declined."""
    from indicatrix_b200 import backend as bk, workloads
    fs = workloads.round_brilliant_frame(8, 8)
    fs.material = materials.tanzanite()
    assert bk.scene_routes_to_gpu(fs)
    m = materials.tanzanite()
    m.anisotropic = 0
    fs.material = m
    assert not bk.scene_routes_to_gpu(fs)
