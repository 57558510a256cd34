"""Writes environment_pins.json: the reference's 180 bit pins of the escape-radiance lookup
(crates/indicatrix/src/optics/raytracer/environment/tests_pins.rs, PINS), one FNV-1a 64
hash per (preset, light pose, observer, head shadow) row in the order its test enumerates
them, with the inputs that test uses.  Run from the repository root with the reference
checked out at ../reference or pass its path."""
import json
import os
import re
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
src = open(os.path.join(ref, "crates/indicatrix/src/optics/raytracer/environment/tests_pins.rs")).read()
block = src[src.index("const PINS: [u64; 180] = ["):src.index("];", src.index("const PINS"))]
pins = [int(m.replace("_", ""), 16) for m in re.findall(r"0x([0-9a-f_]{19})", block)]
assert len(pins) == 180
out = {
    "source": "crates/indicatrix/src/optics/raytracer/environment/tests_pins.rs (PINS, as_lit_is_bit_identical)",
    "presets": ["LightTent", "IsoHemisphere", "WhiteTray", "ShopLights", "WindowDaylight", "DaylightDome",
                "DaylightSun", "Daylight", "Incandescent", "IlluminantA", "RingLights", "DarkSpotlight", "Aset",
                "UvLamp365", "UvLamp395"],
    "preset_index": [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14],
    "exposure": 1.3,
    "poses": [[0.84, 0.94], [-2.1, 0.3]],
    "observer_on": [0.1, 0.95, 0.3],
    "head_shadow_deg": [0.0, 16.0, 30.0],
    "heights": [[0.98, 0.7, 0.35, 0.1], [0.049, 0.02, -0.02, -0.049], [-0.1, -0.35, -0.7, -0.98]],
    "azimuths": [[1.0, 0.0], [0.0, 1.0], [0.6, 0.8], [-0.8, -0.6]],
    "lambdas": [450.0, 550.0, 650.0],
    "pins": ["0x%016x" % p for p in pins],
}
json.dump(out, open(os.path.join(os.path.dirname(__file__), "environment_pins.json"), "w"), indent=1)
