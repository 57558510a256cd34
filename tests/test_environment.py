"""The escape-radiance lookup of every lighting preset against the reference's own bit pins.

tests/golden/environment_pins.json holds the reference's 180 FNV-1a 64 pins of
`sample_environment_channels` (environment/tests_pins.rs, as_lit_is_bit_identical):
each of the 15 presets under two light poses, the observer off and on and three
head-shadow sizes, over 48 directions (above, inside and below the horizon band) at 450,
550 and 650 nm.  The oracle's lookup reproduces every row bit for bit; the product host
code builds each preset's environment record bit-identical to the oracle's; the routing
predicate takes every model the path traces and declines the UV lamps.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from indicatrix_b200 import abi, materials, workloads

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "environment_pins.json")))
FNV_OFFSET, FNV_PRIME = 0xCBF29CE484222325, 0x100000001B3


@pytest.fixture(scope="module")
def oracle():
    from oracle import ix_oracle
    return ix_oracle


def fold(h, bits):
    for b in int(bits).to_bytes(4, "little"):
        h ^= b
        h = (h * FNV_PRIME) & 0xFFFFFFFFFFFFFFFF
    return h


def pin_directions():
    """tests_pins.rs directions(): y per ring, radius = sqrt(mul_add(-y, y, 1)) in f32."""
    out = []
    for group in GOLDEN["heights"]:
        for y in group:
            y = np.float32(y)
            r = np.float32(np.sqrt(np.float32(np.float64(y) * -np.float64(y) + 1.0)))
            for hx, hz in GOLDEN["azimuths"]:
                out.append(np.array([np.float32(hx) * r, y, np.float32(hz) * r], np.float32))
    return out


def observers():
    v = np.array(GOLDEN["observer_on"], np.float32)
    d = np.float32(np.float32(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    return [np.zeros(3, np.float32), (v * (np.float32(1.0) / np.sqrt(d))).astype(np.float32)]


def rows():
    """(preset index, pose, observer, head shadow, pin) in the reference test's order."""
    k = 0
    for idx in GOLDEN["preset_index"]:
        for pose in GOLDEN["poses"]:
            for obs in observers():
                for shadow in GOLDEN["head_shadow_deg"]:
                    yield idx, pose, obs, shadow, int(GOLDEN["pins"][k], 16)
                    k += 1


@pytest.mark.parametrize("preset", range(15))
def test_every_environment_pin(oracle, preset):
    """as_lit_is_bit_identical (environment/tests_pins.rs:301), the preset's 12 rows."""
    f32p = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    dirs = pin_directions()
    assert len(dirs) == 48
    for idx, pose, obs, shadow, pin in rows():
        if idx != preset:
            continue
        env = oracle.environment_preset(idx, GOLDEN["exposure"], pose[0], pose[1], 0.0, 1.0, shadow)
        h = FNV_OFFSET
        for d in dirs:
            for lam in GOLDEN["lambdas"]:
                v = oracle.lib().ixo_environment_channel(C.byref(env), f32p(d), C.c_float(lam), f32p(obs))
                h = fold(h, np.float32(v).view(np.uint32))
        assert h == pin, (GOLDEN["presets"][idx], pose, shadow)


def test_host_environment_records_match_oracle(oracle):
    """ix_environment_preset (product host code) builds every preset's record with the
    oracle's bits, for several poses, trays, glare and head shadows."""
    from indicatrix_b200.backend import environment_preset
    for preset in range(15):
        for yaw, pitch, tray, glare, hs in [(0.85, 0.95, 0.2, 0.7, 16.0), (-2.1, 0.3, 0.0, 1.0, 30.0),
                                            (0.0, -0.2, 0.5, 0.0, 0.0)]:
            a = environment_preset(preset, 1.3, yaw, pitch, tray, glare, hs)
            b = oracle.environment_preset(preset, 1.3, yaw, pitch, tray, glare, hs)
            assert bytes(a) == bytes(b), preset
    with pytest.raises(ValueError):
        environment_preset(15)


def test_routing_of_the_lighting_models():
    """Every lighting model of the reference routes; a UV lamp (fluorescence source,
    gpu_backend/mod.rs:288-298) declines; DaylightSun routes polished, frosted and
    scattering stones (the frosted facets' light samples are traced; a scattering event
    takes none under the analytic sun, scattering/hg_nee.rs:165)."""
    from indicatrix_b200.backend import environment_preset, scene_routes_to_gpu
    fs = workloads.round_brilliant_frame(8, 8)
    for preset in range(13):
        fs.environment = environment_preset(preset, 1.0, 0.5, 0.8)
        assert scene_routes_to_gpu(fs), preset
    for preset in (13, 14):
        fs.environment = environment_preset(preset, 1.0, 0.5, 0.8)
        assert not scene_routes_to_gpu(fs), preset
    fs.environment = environment_preset(6, 1.0, 0.5, 0.8)
    fin = np.zeros(fs.planes.shape[0], np.uint8)
    fs.facet_finishes = fin
    assert scene_routes_to_gpu(fs)
    fin[40] = 1
    assert scene_routes_to_gpu(fs)
    fs.facet_finishes = None
    fs.material = materials.with_scattering(materials.diamond(), 1.0, 0.3)
    assert scene_routes_to_gpu(fs)
