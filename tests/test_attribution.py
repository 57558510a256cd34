"""Spectral attribution on the CPU: the oracle's event recorder and classifier against the
reference's own tests, and the host attribution map against attribution_map.rs's tests.

The cases quote crates/indicatrix/src/color/metrics/attribution.rs (tests module),
optics/raytracer/transport/path_events.rs (tests), transport/tests/attribution_tests.rs
and renderer/attribution_map.rs (tests); each test names the one it restates.
"""
import struct

import numpy as np
import pytest

from indicatrix_b200 import abi, materials
from indicatrix_b200.attribution import (AttributionMap, energy_error, energy_share, probability_error,
                                         probability_share)

PRESET_ISO_HEMISPHERE = 1
PRESET_RING_LIGHTS = 10
YAW, PITCH = 0.85, 0.95


def bits3(v):
    return [struct.unpack("<I", struct.pack("<f", float(x)))[0] for x in v]


def glam_normalize(v):
    v = np.asarray(v, np.float32)
    d = np.float32(np.float32(v[0] * v[0] + v[1] * v[1]) + np.float32(v[2] * v[2]))
    return (v * (np.float32(1.0) / np.sqrt(d))).astype(np.float32)


def srb_scene(oracle, material, preset, max_bounces=12, glare=1.0):
    import ctypes as C

    planes = np.ascontiguousarray(oracle.standard_round_brilliant())
    sc = abi.Scene()
    sc.planes = planes.ctypes.data_as(C.POINTER(C.c_float))
    sc.n_planes = planes.shape[0]
    sc.material = material
    sc.max_bounces = max_bounces
    sc.environment = oracle.environment_preset(preset, 1.0, YAW, PITCH, 0.0, glare)
    return sc, planes


def centred(oracle, i, salt):
    """attribution_tests.rs:22: a uniform [-0.5, 0.5) draw, in f32."""
    h = np.float32(oracle.lib().ixo_hash_u32((i ^ salt) & 0xFFFFFFFF))
    return np.float32(np.float32(h / np.float32(4294967295.0)) - np.float32(0.5))


def ray_for(oracle, i):
    """attribution_tests.rs:27: an oblique camera ray from above that mostly meets the stone."""
    f = np.float32
    origin = np.array([centred(oracle, i, 0x1111) * f(1.4), 2.5, centred(oracle, i, 0x2222) * f(1.4)], np.float32)
    d = glam_normalize([centred(oracle, i, 0x3333) * f(0.8), -1.0, centred(oracle, i, 0x4444) * f(0.8)])
    return origin, d


def seed_and_hero(oracle, i):
    """attribution_tests.rs:35."""
    seed = 9000 + i
    return seed, float(np.float32(np.float32(oracle.lib().ixo_hash_u32(seed)) / np.float32(4294967295.0)))


# --- color/metrics/attribution.rs tests -------------------------------------------------

def exiting(oracle, normal, direction):
    ev = oracle.path_events()
    ev.first_facet, ev.first_entered = 0, 1
    ev.exit_facet = 1
    ev.exit_normal[:] = [float(x) for x in normal]
    ev.exit_dir[:] = [float(x) for x in glam_normalize(direction)]
    ev.exit_bounce = 2
    ev.termination = oracle.TERM_ESCAPED
    return ev


def classify(oracle, ev, observer):
    return oracle.classify_path(ev, observer, PRESET_ISO_HEMISPHERE, YAW, PITCH)


def test_a_path_with_no_facet_event_is_a_miss(oracle):
    assert classify(oracle, oracle.path_events(), [0, 0, 1]) == abi.CLASS_MISS


def test_an_outside_reflection_is_glare_whatever_happened_after(oracle):
    ev = oracle.path_events()
    ev.first_facet, ev.first_entered = 4, 0
    ev.termination = oracle.TERM_ESCAPED
    assert classify(oracle, ev, [0, 0, 1]) == abi.CLASS_GLARE


def test_exits_follow_the_analytical_predicates(oracle):
    windowed = exiting(oracle, [0, -1, 0], [0.1, 1.0, 0.0])
    assert classify(oracle, windowed, [0, 0, 1]) == abi.CLASS_WINDOWED
    returned = exiting(oracle, [0, 1, 0], [0.3, 0.9, 0.0])
    assert classify(oracle, returned, [0, 0, 1]) == abi.CLASS_RETURNED
    assert classify(oracle, returned, list(returned.exit_dir)) == abi.CLASS_SHADOW
    side = exiting(oracle, [1, 0, 0], [1.0, 0.0, 0.0])
    assert classify(oracle, side, [0, 0, 1]) == abi.CLASS_SIDE_EXIT


def test_paths_that_never_exit_are_labelled_by_how_they_stopped(oracle):
    def stopped(termination):
        ev = oracle.path_events()
        ev.first_facet, ev.first_entered = 0, 1
        ev.termination = termination
        return classify(oracle, ev, [0, 0, 1])

    assert stopped(oracle.TERM_CAP) == abi.CLASS_BUDGET
    assert stopped(oracle.TERM_RR) == abi.CLASS_KILLED
    assert stopped(oracle.TERM_ESCAPED) == abi.CLASS_NO_INTERSECTION
    assert stopped(7) == abi.CLASS_NO_INTERSECTION  # no termination recorded: Invalid


def test_unlit_exit_under_the_studio_rig(oracle):
    """An upward exit away from every light of the ring rig is InsufficientIllumination
    (visibility.rs:64), toward the key light it is returned."""
    ev = exiting(oracle, [0, 1, 0], [0.0, 0.06, -1.0])
    lit = oracle.metrics_lighting(PRESET_RING_LIGHTS, YAW, PITCH)
    assert lit[0] > 0
    cls = oracle.classify_path(ev, [0, 0, 1], PRESET_RING_LIGHTS, YAW, PITCH)
    assert cls in (abi.CLASS_UNLIT, abi.CLASS_RETURNED)
    key = glam_normalize([np.cos(PITCH) * np.sin(YAW), np.sin(PITCH), np.cos(PITCH) * np.cos(YAW)])
    ev_key = exiting(oracle, [0, 1, 0], key)
    assert oracle.classify_path(ev_key, [0, 0, 1], PRESET_RING_LIGHTS, YAW, PITCH) == abi.CLASS_RETURNED


# --- optics/raytracer/transport/path_events.rs tests ------------------------------------

def test_an_outside_reflection_is_a_first_facet_that_did_not_enter(oracle):
    ev = oracle.path_events()
    oracle.path_events_facet(ev, 0, 3, [0, 1, 0], False, False, [0, 1, 0])
    assert (ev.first_facet, ev.first_entered) == (3, 0)
    assert ev.exit_facet == -1


def test_entry_reflections_exit_and_reentry_are_told_apart(oracle):
    ev = oracle.path_events()
    f = oracle.path_events_facet
    f(ev, 0, 1, [0, 1, 0], False, True, [0, -1, 0])
    f(ev, 1, 2, [0, -1, 0], True, True, [0, 1, 0])
    f(ev, 2, 4, [1, 0, 0], True, False, [1, 0, 0])
    f(ev, 3, 5, [0, 0, 1], False, True, [0, 0, 1])
    f(ev, 4, 6, [1, 0, 0], True, True, [0, 0, 1])
    f(ev, 5, 7, [1, 0, 0], True, False, [1, 0, 0])
    assert (ev.first_facet, ev.first_entered) == (1, 1)
    assert (ev.exit_facet, ev.exit_bounce) == (4, 2)
    assert ev.bounces_before_exit == 1
    assert ev.reentered == 1


# --- transport/tests/attribution_tests.rs ----------------------------------------------

@pytest.mark.parametrize("material", ["diamond", "sapphire", "absorbing"])
def test_attributed_radiance_equals_plain_radiance(oracle, material):
    """attribution_tests.rs:87: the recorder only observes (the same XYZ bits)."""
    mat = {"diamond": materials.diamond(), "sapphire": materials.sapphire(),
           "absorbing": materials.isotropic(materials.diamond().dispersion,
                                            spline_alpha=np.linspace(0.5, 3.0, 16, dtype=np.float32))}[material]
    sc, _keep = srb_scene(oracle, mat, PRESET_RING_LIGHTS)
    for i in range(0, 3334, 7):
        o, d = ray_for(oracle, i)
        seed, hero = seed_and_hero(oracle, i)
        plain, _ = oracle.trace_ray(sc, o, d, seed, hero)
        attributed, _ev = oracle.trace_ray_events(sc, o, d, seed, hero)
        assert bits3(plain) == bits3(attributed), (material, i)


def test_a_convex_stone_never_reenters_and_rarely_loses_a_path_after_entry(oracle):
    """attribution_tests.rs:117: no re-entry, a termination for every entered path, and at
    most 2 % of entered paths lost (no intersection inside a convex stone)."""
    sc, _keep = srb_scene(oracle, materials.diamond(), PRESET_ISO_HEMISPHERE)
    entered = lost = 0
    for i in range(4000):
        o, d = ray_for(oracle, i)
        seed, hero = seed_and_hero(oracle, i)
        _, ev = oracle.trace_ray_events(sc, o, d, seed, hero)
        assert ev.reentered == 0, i
        cls = oracle.classify_path(ev, -d, PRESET_ISO_HEMISPHERE, YAW, PITCH)
        lost += cls == abi.CLASS_NO_INTERSECTION
        if ev.first_facet >= 0 and ev.first_entered:
            entered += 1
            assert ev.termination in (oracle.TERM_ESCAPED, oracle.TERM_RR, oracle.TERM_CAP)
    assert entered > 200
    assert lost * 50 <= entered, (lost, entered)


def test_roulette_and_scatter_are_reasons(oracle):
    """russian_roulette_and_scatter_are_reasons (attribution_tests.rs:201): a scattering,
    absorbing corundum (sigma_s 3, g 0.5; the sapphire builder stands in for the built-in
    ruby) at a 64-bounce budget scatters, ends paths by roulette and by scattering
    absorption, and labels every entered path that never exited by its termination."""
    mat = materials.with_scattering(materials.sapphire(), 3.0, 0.5)
    sc, _keep = srb_scene(oracle, mat, PRESET_ISO_HEMISPHERE, max_bounces=64)
    roulette = absorbed = scattered = 0
    expected = {oracle.TERM_RR: abi.CLASS_KILLED, oracle.TERM_SCATTER_ABSORBED: abi.CLASS_KILLED,
                oracle.TERM_CAP: abi.CLASS_BUDGET}
    for i in range(3000):
        o, d = ray_for(oracle, i)
        seed, hero = seed_and_hero(oracle, i)
        _, ev = oracle.trace_ray_events(sc, o, d, seed, hero)
        scattered += ev.scattered
        roulette += ev.termination == oracle.TERM_RR
        absorbed += ev.termination == oracle.TERM_SCATTER_ABSORBED
        if ev.exit_facet < 0 and ev.first_facet >= 0 and ev.first_entered:
            cls = oracle.classify_path(ev, -d, PRESET_ISO_HEMISPHERE, YAW, PITCH)
            assert cls == expected.get(ev.termination, abi.CLASS_NO_INTERSECTION), i
    assert scattered > 0 and absorbed > 0 and roulette > 0, (scattered, absorbed, roulette)


def test_a_missing_ray_records_only_the_escape(oracle):
    """attribution_tests.rs:150."""
    sc, _keep = srb_scene(oracle, materials.diamond(), PRESET_ISO_HEMISPHERE)
    d = np.array([0, 1, 0], np.float32)
    seed, hero = seed_and_hero(oracle, 1)
    _, ev = oracle.trace_ray_events(sc, [0, 2.5, 0], d, seed, hero)
    assert ev.first_facet == -1 and ev.exit_facet == -1
    assert ev.has_escaped_dir == 1 and bits3(ev.escaped_dir) == bits3(d)
    assert ev.termination == oracle.TERM_ESCAPED
    assert oracle.classify_path(ev, -d, PRESET_ISO_HEMISPHERE, YAW, PITCH) == abi.CLASS_MISS


def test_glare_is_bounce_zero_outside(oracle):
    """attribution_tests.rs:166: surface glare scales only the outside reflection."""
    d = glam_normalize([0.18, -1.0, 0.07])
    o = np.array([0, 2.5, 0], np.float32)

    def run(glare):
        sc, _keep = srb_scene(oracle, materials.diamond(), PRESET_ISO_HEMISPHERE, glare=glare)
        glare_y, count, classes = np.float32(0.0), 0, []
        for i in range(512):
            seed, hero = seed_and_hero(oracle, i)
            xyz, ev = oracle.trace_ray_events(sc, o, d, seed, hero)
            cls = oracle.classify_path(ev, -d, PRESET_ISO_HEMISPHERE, YAW, PITCH)
            if cls == abi.CLASS_GLARE:
                glare_y = np.float32(glare_y + xyz[1])
                count += 1
            classes.append(cls)
        return glare_y, count, classes

    full_y, full_n, full_c = run(1.0)
    none_y, none_n, none_c = run(0.0)
    assert full_n > 0 and full_y > 0.0
    assert none_y <= 1e-6
    assert full_n == none_n and full_c == none_c


# --- renderer/attribution_map.rs tests --------------------------------------------------

def map_with_samples():
    m = AttributionMap(2, 2)
    m.add(0, abi.CLASS_RETURNED, 2.0)
    m.add(0, abi.CLASS_WINDOWED, 1.0)
    m.add(0, abi.CLASS_MISS, 5.0)
    m.add(1, abi.CLASS_KILLED, 0.5, scattered=True)
    m.add(3, abi.CLASS_GLARE, float("nan"))
    return m


def test_an_invalid_size_gives_an_empty_map_that_ignores_samples():
    for w, h in [(0, 4), (4, 0), (2000, 2000)]:
        assert AttributionMap.checked(w, h) is None
        m = AttributionMap(w, h)
        assert m.pixels.size == 0
        m.add(0, abi.CLASS_RETURNED, 1.0)
        assert int(m.totals()["samples"]) == 0
    assert AttributionMap.checked(1024, 1024) is not None


def test_classes_conserve_hits():
    m = map_with_samples()
    for p in m.pixels:
        assert int(p["counts"].sum()) == int(p["hits"])
    t = m.totals()
    assert (int(t["samples"]), int(t["hits"])) == (5, 4)
    delivered = np.float32(0.0)
    for v in t["y_sum"]:
        delivered = np.float32(delivered + v)
    assert abs(delivered - 3.5) <= 1e-6 * 3.5
    assert int(t["scattered"]) == 1


def test_a_non_finite_luminance_is_counted_but_not_summed():
    p = map_with_samples().pixels[3]
    assert int(p["counts"][abi.CLASS_GLARE]) == 1
    assert bits3([p["y_sum"][abi.CLASS_GLARE]]) == bits3([0.0])


def test_shares_sum_to_one_and_errors():
    p = map_with_samples().pixels[0]
    prob = sum(float(probability_share(p, k)) for k in range(abi.ATTRIBUTION_CLASSES))
    energy = sum(float(energy_share(p, k)) for k in range(abi.ATTRIBUTION_CLASSES))
    assert abs(prob - 1.0) <= 1e-6 and abs(energy - 1.0) <= 1e-6
    assert abs(energy_share(p, abi.CLASS_RETURNED) - 2.0 / 3.0) <= 1e-6
    empty = np.zeros((), abi.attribution_dtype())
    for fn in (probability_share, energy_share, probability_error, energy_error):
        assert fn(empty, abi.CLASS_RETURNED) == 0.0


def test_the_standard_errors_follow_the_textbook_forms():
    m = AttributionMap(1, 1)
    for y in [1.0, 3.0, 1.0, 3.0]:
        m.add(0, abi.CLASS_RETURNED, y)
    assert probability_error(m.pixels[0], abi.CLASS_RETURNED) == 0.0
    assert abs(energy_error(m.pixels[0], abi.CLASS_RETURNED) - np.sqrt(np.float32(1.0 / 3.0))) <= 1e-5
    m.add(0, abi.CLASS_WINDOWED, 1.0)
    assert abs(probability_error(m.pixels[0], abi.CLASS_RETURNED) - np.sqrt(np.float32(0.8 * 0.2 / 5.0))) <= 1e-6


def test_clear_forgets_the_samples_and_keeps_the_size():
    m = map_with_samples()
    m.clear()
    assert (m.width, m.height, m.pixels.size) == (2, 2, 4)
    assert int(m.totals()["samples"]) == 0


def test_oracle_add_matches_the_host_map(oracle):
    """The oracle's AttributionPixel::add and the host map's, bit for bit."""
    rng = np.random.default_rng(5)
    host = AttributionMap(1, 1)
    ora = np.zeros(1, abi.attribution_dtype())
    for _ in range(400):
        cls = int(rng.choice([abi.CLASS_MISS] + list(range(9))))
        y = float(np.float32(rng.gamma(0.5, 2.0))) if rng.random() > 0.02 else float("inf")
        host.add(0, cls, y)
        oracle.attribution_add(ora, 0, cls, y)
    assert host.pixels.tobytes() == ora.tobytes()


# --- the attributed frame loop ---------------------------------------------------------

def test_attributed_frame_matches_the_plain_frame(oracle):
    """Per-pixel XYZ sums of the attributed loop equal the plain loop's bit for bit; every
    sample is counted; classes conserve hits; a second call continues the sums in sample
    order (two halves equal one whole)."""
    from indicatrix_b200 import workloads

    fs = workloads.round_brilliant_frame(32, 32, max_bounces=16)
    sc = fs.to_abi()
    light = abi.MetricsLighting(PRESET_ISO_HEMISPHERE, 0.0, 0.0, 20.0)
    n = 32 * 32
    m, sums, dropped = oracle.attribute_pixels(sc, light, 0, n, 0, 8, threads=4)
    plain = oracle.trace_pixels(sc, 0, n, 0, 8, threads=4)
    assert sums.tobytes() == plain.tobytes()
    assert dropped == 0
    assert (m["samples"] == 8).all()
    assert (m["counts"].sum(axis=1) == m["hits"]).all()
    assert m["hits"].sum() > 0 and (m["counts"][:, abi.CLASS_RETURNED].sum() > 0)
    m2, _, _ = oracle.attribute_pixels(sc, light, 0, n, 0, 4, threads=4)
    m2, _, _ = oracle.attribute_pixels(sc, light, 0, n, 4, 4, threads=4, pixel_map=m2)
    assert m2.tobytes() == m.tobytes()


# --- the convex-exit shortcut of the device's bounce loop ----------------------------

def test_a_ray_leaving_through_a_facet_misses_the_stone(oracle):
    """The device skips the plane scan for a ray that starts more than 1e-6 outside the
    half-space of the facet it left and moves away from it (denom > 1e-6).  The oracle's
    scan (the reference's slab arithmetic) must report a miss for every such ray: exit
    points of rays from inside the round brilliant, the step cut and random stones, with
    outward directions down to grazing, restarted 1e-4 along the direction as the
    bounce loop restarts them."""
    import ctypes as C

    from indicatrix_b200 import geometry

    lib = oracle.lib()
    t, f = C.c_float(), C.c_int32()
    stones = [np.ascontiguousarray(oracle.standard_round_brilliant()), geometry.to_f32(geometry.step_cut())]
    from indicatrix_b200 import workloads

    stones += [np.ascontiguousarray(s.planes, np.float32) for s in workloads.random_stones(3, seed=11)]
    rng = np.random.default_rng(3)
    f32 = np.float32
    checked = skipped = 0
    for planes in stones:
        planes = np.ascontiguousarray(planes, np.float32)
        centre = np.array([0.0, -0.1, 0.0], np.float32)
        for _ in range(600):
            d_in = glam_normalize(rng.normal(size=3))
            if not lib.ixo_intersect(oracle._f32p(planes), planes.shape[0], oracle._f32p(centre),
                                     oracle._f32p(d_in), C.byref(t), C.byref(f)):
                continue
            fi = f.value
            h = (centre + f32(t.value) * d_in).astype(np.float32)
            n = planes[fi, :3]
            # An outward direction: a random unit vector flipped to the facet's side, some
            # of them nearly grazing.
            d = glam_normalize(rng.normal(size=3))
            if f32(np.dot(n, d)) < 0:
                d = -d
            if rng.random() < 0.3:
                d = glam_normalize(d - n * f32(np.dot(n, d) * f32(0.999)))
            o = (h + d * f32(1e-4)).astype(np.float32)
            p = planes[fi]
            denom = f32(f32(f32(p[0] * d[0]) + f32(p[1] * d[1])) + f32(p[2] * d[2]))
            side = f32(p[3] + f32(f32(f32(p[0] * o[0]) + f32(p[1] * o[1])) + f32(p[2] * o[2])))
            if not (denom > 1e-6 and side > 1e-6):
                skipped += 1
                continue
            checked += 1
            hit = lib.ixo_intersect(oracle._f32p(planes), planes.shape[0], oracle._f32p(o), oracle._f32p(d),
                                    C.byref(t), C.byref(f))
            assert hit == 0, (fi, o, d, t.value, f.value)
    assert checked > 2000 and skipped > 0
