"""Next-event estimation toward the DaylightSun disc at frosted facets, in the oracle.

The reference's own checks (optics/raytracer/scattering/tests.rs:672-850) restated on
the oracle: the disc draws are unit vectors inside the 0.27 degree disc, uniform in solid
angle, with the constant pdf the independent lookup also returns (zero outside); the
balance weights of the two techniques sum to one and together conserve a Lambertian
reflector's energy; one frosted-exterior deposit equals the analytic direct-light value
(cos / pi) x solid angle x L_sun(lambda) and a surface facing away gets none.  Beside
them: the shadow probe of a carved stone, and the routing, which traces frosted and
scattering stones under the sun.
"""
import ctypes as C
import math

import numpy as np
import pytest

from indicatrix_b200 import geometry, materials, workloads

DISC_COS = np.float32(0.9999889)
OMEGA = float(np.float32(2.0 * np.pi) * (np.float32(1.0) - DISC_COS))


@pytest.fixture(scope="module")
def oracle():
    from oracle import ix_oracle
    return ix_oracle


def f32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def sun(oracle):
    """The tests' sun: DaylightSun at exposure 1.3, light yaw 0.4, pitch 1.2."""
    env = oracle.environment_preset(6, 1.3, 0.4, 1.2)
    return env, np.array(env.key_dir[:3], np.float32)


def draw(oracle, env, u0, u1):
    d = np.zeros(3, np.float32)
    pdf = oracle.lib().ixo_sun_nee_sample(C.byref(env), u0, u1, f32p(d))
    return d, np.float32(pdf)


def test_sun_draws_are_uniform_over_the_disc_with_the_matching_pdf(oracle):
    """sun_nee_draws_are_uniform_over_the_disc_with_the_matching_pdf (tests.rs:672)."""
    env, key = sun(oracle)
    grid, inner = 64, 0
    half = np.float32(np.float32(1.0) - (np.float32(1.0) - DISC_COS) * np.float32(0.5))
    for i in range(grid):
        for j in range(grid):
            u0 = float(np.float32((i + 0.5) / grid))
            u1 = float(np.float32((j + 0.5) / grid))
            d, pdf = draw(oracle, env, u0, u1)
            assert abs(float(np.linalg.norm(d.astype(np.float64))) - 1.0) < 1e-5
            c = np.float32(np.dot(d, key))
            assert c >= DISC_COS - np.float32(2e-7), (u0, u1, c)
            assert abs(float(pdf) * OMEGA - 1.0) < 1e-3
            assert np.float32(oracle.lib().ixo_sun_nee_pdf(C.byref(env), f32p(d))).view(np.uint32) == \
                pdf.view(np.uint32)
            inner += int(c >= half)
    assert abs(inner / grid**2 - 0.5) < 0.04
    # 0.4 degrees off the key is outside the disc.
    perp = np.cross(key, [0.0, 1.0, 0.0] if abs(key[0]) > 0.9 else [1.0, 0.0, 0.0])
    perp /= np.linalg.norm(perp)
    a = math.radians(0.4)
    out = (key * math.cos(a) + perp * math.sin(a)).astype(np.float32)
    assert oracle.lib().ixo_sun_nee_pdf(C.byref(env), f32p(out / np.linalg.norm(out))) == 0.0


def test_mis_weights_sum_to_one_and_conserve_energy(oracle):
    """sun_mis_weights_sum_to_one_and_the_two_techniques_conserve_energy (tests.rs:741):
    a Lambertian reflector facing the sun, both techniques' expectations over a
    stratified disc grid sum to L_sun x solid angle x cos / pi."""
    env, key = sun(oracle)
    bh = oracle.lib().ixo_balance_heuristic
    grid, nee, bsdf = 64, 0.0, 0.0
    for i in range(grid):
        for j in range(grid):
            d, p_light = draw(oracle, env, float(np.float32((i + 0.5) / grid)), float(np.float32((j + 0.5) / grid)))
            c = np.float32(np.dot(d, key))
            assert c > 0
            p_bsdf = np.float32(c / np.float32(np.pi))
            w_nee, w_bsdf = bh(float(p_light), float(p_bsdf)), bh(float(p_bsdf), float(p_light))
            assert abs(w_nee + w_bsdf - 1.0) < 1e-6
            nee += w_nee * float(p_bsdf) * 40000.0
            bsdf += w_bsdf * float(p_bsdf) * 40000.0
    omega = 1.0 / float(p_light)
    total = (nee + bsdf) / grid**2 * omega
    target = 1.0 / math.pi * omega * 40000.0
    assert abs(total / target - 1.0) < 1e-3
    assert bsdf / nee < 1e-3


def deposit(oracle, fs, origin, normal, seed, bounce=3, lambdas=None):
    lam = lambdas if lambdas is not None else (np.float32(40.0) * np.arange(8, dtype=np.float32) +
                                               np.float32(420.0)).astype(np.float32)
    rad = np.zeros(8, np.float32)
    sc = fs.to_abi()
    oracle.lib().ixo_frosted_sun_nee(C.byref(sc), f32p(np.asarray(origin, np.float32)),
                                     f32p(np.asarray(normal, np.float32)), seed, bounce, f32p(lam),
                                     f32p(np.ones(8, np.float32)), f32p(rad))
    return lam, rad


def test_frosted_exterior_deposit_is_the_analytic_sun_value(oracle):
    """frosted_exterior_nee_deposits_the_analytic_sun_value (tests.rs:804): facing the
    sun, each channel receives (1 / pi) x solid angle x 40 000 x spd x exposure within
    2e-3; facing away, nothing."""
    env, key = sun(oracle)
    fs = workloads.round_brilliant_frame(8, 8)
    fs.environment = env
    for seed in range(32):
        lam, rad = deposit(oracle, fs, (0.0, 0.0, 0.0), key, oracle.lib().ixo_hash_u32(seed))
        for k in range(8):
            expected = (1.0 / math.pi) * OMEGA * 40000.0 * oracle.lib().ixo_d65(float(lam[k])) * 1.3
            assert abs(float(rad[k]) / expected - 1.0) < 2e-3, (seed, k)
    _, dark = deposit(oracle, fs, (0.0, 0.0, 0.0), -key, 7)
    assert np.all(dark == 0.0)


def test_carved_stone_shadow_probe(oracle):
    """On a carved stone the light sample is shadow-probed (frosted.rs:128): from the
    stone's centre the sun's direction runs into the crown (no deposit), from above the
    stone it escapes (a deposit); on an uncarved stone there is no probe."""
    env, key = sun(oracle)
    fs = workloads.round_brilliant_frame(8, 8)
    fs.environment = env
    _, free = deposit(oracle, fs, (0.0, 0.0, 0.0), key, 11)
    assert np.all(free > 0.0)
    fs.tools = [geometry.tool_ball((0.9, 0.0, 0.0), 0.05)]
    _, blocked = deposit(oracle, fs, (0.0, 0.0, 0.0), key, 11)
    assert np.all(blocked == 0.0)
    _, above = deposit(oracle, fs, (0.0, 2.0, 0.0), key, 11)
    assert np.array_equal(above, free)


def test_routing_under_the_sun():
    """DaylightSun routes a frosted stone (its light samples are traced), carved or not,
    and a scattering one (a Henyey-Greenstein event takes no light sample under the
    analytic sun, scattering/hg_nee.rs:165)."""
    from indicatrix_b200.backend import environment_preset, scene_routes_to_gpu
    fs = workloads.round_brilliant_frame(8, 8)
    fs.environment = environment_preset(6, 1.0, 0.5, 0.8)
    fin = np.zeros(fs.planes.shape[0], np.uint8)
    fin[40] = 1
    fs.facet_finishes = fin
    assert scene_routes_to_gpu(fs)
    fs.tools = [geometry.tool_ball((0.0, 0.32, 0.0), 0.22)]
    assert scene_routes_to_gpu(fs)
    fs.material = materials.with_scattering(materials.diamond(), 1.0, 0.3)
    assert scene_routes_to_gpu(fs)
