"""Frosted (bruted) facets in the CPU oracle: apply_frosted_bounce
(optics/raytracer/scattering/frosted.rs:289) against the reference's own furnace tests.

The reference holds no golden bits for a frosted facet that travel off Windows (its pin
hashes, renderer/gpu/pin_tests.rs:160, are Windows-only); the pins here are its
energy-conservation anchors: tests/raytracer_tests/material_equivalence_finish.rs:156
(frosted girdle, isotropic) and white_furnace_energy_conservation.rs:190 (frosted girdle,
birefringent), each to its own 0.025 relative tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from indicatrix_b200 import abi, materials

L0 = 2.5
GIRDLE = range(33, 49)  # STANDARD_ROUND_BRILLIANT_GIRDLE_FACETS (geometry/cuts/round_brilliant.rs:22)


def bruted_girdle_finishes(n):
    """fixtures.rs:16: Polished everywhere except the girdle band, which is Frosted."""
    f = np.zeros(n, np.uint8)
    f[list(GIRDLE)] = 1
    return f


def furnace_scene(oracle, material, finishes=True, max_bounces=12):
    planes = np.ascontiguousarray(oracle.standard_round_brilliant())
    fin = bruted_girdle_finishes(planes.shape[0])
    sc = abi.Scene()
    sc.camera = oracle.camera_new(0.35, 0.28, 5.0, 18.0)
    sc.width = sc.height = 12
    sc.planes = planes.ctypes.data_as(C.POINTER(C.c_float))
    sc.n_planes = planes.shape[0]
    if finishes:
        sc.facet_finishes = fin.ctypes.data_as(C.POINTER(C.c_uint8))
        sc.n_finishes = fin.shape[0]
    sc.material = material
    sc.max_bounces = max_bounces
    sc.environment = oracle.environment_uniform(L0)
    return sc, (planes, fin)


def furnace_target(oracle):
    out = np.zeros(3, np.float32)
    target = np.zeros(3)
    for lam in range(380, 781):
        oracle.lib().ixo_cmf(float(lam), oracle._f32p(out))
        target += out * L0
    return target / 106.856


@pytest.mark.parametrize("birefringent", [False, True], ids=["isotropic", "birefringent"])
def test_frosted_girdle_white_furnace(oracle, birefringent):
    """A colourless, non-dispersive stone (n 1.5, birefringence 0.03 for the second case)
    with a bruted girdle in a uniform environment returns the environment's own radiance,
    within the reference's 0.025 (96 samples per pixel of the 12 x 12 furnace grid, depth
    12).  Frosted events must occur: the same frame with the girdle polished differs."""
    disp = materials.cauchy(1.5, 0.0, 0.0)
    mat = materials.uniaxial(disp, 0.03) if birefringent else materials.isotropic(disp)
    sc, _keep = furnace_scene(oracle, mat)
    _, s64, dropped = oracle.trace_frame(sc, 0, 96, threads=0)
    assert dropped == 0
    mean = s64.reshape(-1, 3).sum(axis=0) / (12 * 12 * 96)
    target = furnace_target(oracle)
    assert np.all(np.abs(mean - target) / target <= 0.025), (mean, target)
    polished, _keep2 = furnace_scene(oracle, mat, finishes=False)
    _, p64, _ = oracle.trace_frame(polished, 0, 96, threads=0)
    assert not np.array_equal(s64, p64)


def test_frosted_entry_scatters_the_path(oracle):
    """A ray entering girdle facet 40 along its inward normal: through a polished facet
    every seed refracts straight across the stone to the same far facet; through the
    frosted one the cosine lobe sends the seeds to many different facets."""
    from test_attribution import glam_normalize

    def exit_facets(finishes):
        sc, keep = furnace_scene(oracle, materials.isotropic(materials.cauchy(1.5, 0.0, 0.0)),
                                 finishes=finishes, max_bounces=2)
        planes = keep[0]
        n = planes[40, :3].astype(np.float64)
        origin = (-planes[40, 3] * n + 0.5 * n).astype(np.float32)
        d = glam_normalize(-n)
        seen = set()
        for seed in range(60):
            _, ev = oracle.trace_ray_events(sc, origin, d, 1000 + seed, 0.37)
            assert ev.first_facet == 40
            if ev.first_entered and ev.exit_facet >= 0:
                seen.add(ev.exit_facet)
        return seen

    assert len(exit_facets(False)) <= 2
    assert len(exit_facets(True)) >= 4  # measured: 6 distinct exits over the 60 seeds
