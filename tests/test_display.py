"""The display pipeline after the path, oracle side (no GPU): the guide-buffer prepass,
the edge-avoiding A-Trous denoiser and the tone-map, pinned to the reference's own
golden fingerprints and behaviour tests:

* tonemap_accumulation_output_is_pinned (renderer/tonemap.rs:427-451): FNV-1a 64 of
  the RGBA8 of an 8x5 xorshift buffer at 16 spp, per color space;
* denoised_output_is_pinned_to_the_pre_move_gui_code (renderer/frame_denoise.rs:232):
  guides of a 24x16 standard round brilliant at (0.60, 0.45, 2.4, 42 deg), 3 spp,
  denoise + sRGB tone-map, FNV-1a 64;
* denoise_and_tonemap_frame_is_identity_at_high_sample_counts (frame_denoise.rs:310);
* the guide-pass signature tests (renderer/guide_pass/tests.rs:167-236);
* a_constant_signature_is_bit_identical_to_none (denoise/mod.rs tests).
"""
import numpy as np
import pytest

from indicatrix_b200 import abi

TONEMAP_PINS = {
    abi.COLOR_SPACE_SRGB: 0x74AAB8AA51E187E5,
    abi.COLOR_SPACE_DISPLAY_P3: 0xDCF971D4DBD5C9D9,
    abi.COLOR_SPACE_REC2020: 0x4855A258E2398CF4,
    abi.COLOR_SPACE_ACESCG: 0x1F4F8288D9889085,
}
FRAME_PIN = 0x4B0EFD3C897E809C
PIN_POSE = (0.60, 0.45, 2.4, 42.0)


def xorshift_f32(seed: int, n: int) -> np.ndarray:
    """The reference tests' Xorshift32::next_f32: (u32 as f64 / u32::MAX as f64) as f32."""
    x = seed if seed else 0xDEADBEEF
    out = np.zeros(n, np.float32)
    for i in range(n):
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        out[i] = np.float32(np.float64(x) / np.float64(0xFFFFFFFF))
    return out


def irregular_colors(n: int, seed: int) -> np.ndarray:
    """tonemap.rs tests' irregular_colors: three draws x 4 per pixel."""
    return (xorshift_f32(seed, 3 * n) * np.float32(4.0)).reshape(n, 3)


def fnv1a64(data: bytes) -> int:
    h = 0xCBF29CE484222325
    for c in data:
        h = ((h ^ c) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def pin_accum(width: int = 24, height: int = 16) -> np.ndarray:
    """frame_denoise.rs tests' pin_accum."""
    i = np.arange(width * height)
    return np.stack([((i * 37) % 101).astype(np.float32) * np.float32(0.03),
                     ((i * 53) % 97).astype(np.float32) * np.float32(0.02),
                     ((i * 71) % 89).astype(np.float32) * np.float32(0.025)], axis=1).reshape(height, width, 3)


def pin_guides(oracle, width=24, height=16, n_d=0.0, pose=PIN_POSE):
    cam = oracle.camera_new(*pose)
    return oracle.generate_guide_buffers(width, height, cam, oracle.standard_round_brilliant(), n_d)


@pytest.mark.parametrize("space", sorted(TONEMAP_PINS))
def test_tonemap_accumulation_is_pinned(oracle, space):
    accum = irregular_colors(40, 0x13579BDF).reshape(5, 8, 3)
    rgba = oracle.tonemap_accumulation(accum, 16, space)
    assert fnv1a64(rgba.tobytes()) == TONEMAP_PINS[space]


def test_denoised_frame_is_pinned(oracle):
    depth, normal, facet, _ = pin_guides(oracle)
    rgba = oracle.denoise_and_tonemap_frame(pin_accum(), 3, depth, normal, facet, None)
    assert fnv1a64(rgba.tobytes()) == FRAME_PIN
    # The fixture is filtered, not the taper's identity copy.
    raw = oracle.tonemap_to_rgba(pin_accum(), float(np.float32(1.0) / np.float32(3.0)))
    assert not np.array_equal(rgba, raw)


def test_identity_at_high_sample_counts(oracle):
    """taper(50000) < 0.02: the frame is the tone-mapped average, bit for bit."""
    w, h, spp = 6, 5, 50_000
    x = (np.arange(w * h) % w).astype(np.float32)
    # 0.1f32.mul_add(-x, 2.0): the f64 product and sum are exact for x < 6, so rounding
    # them once to f32 is the fused result.
    accum = np.stack([np.float32(1.0) + x, np.float32(0.5) * x,
                      (np.float64(np.float32(0.1)) * -x.astype(np.float64) + 2.0).astype(np.float32)],
                     axis=1).reshape(h, w, 3).astype(np.float32)
    depth = (np.arange(w * h, dtype=np.float32) * np.float32(0.01) + np.float32(1.0)).reshape(h, w)
    normal = np.tile(np.array([0.0, 1.0, 0.0], np.float32), (h, w, 1))
    facet = (np.arange(w * h) % w).astype(np.int32).reshape(h, w)
    got = oracle.denoise_and_tonemap_frame(accum, spp, depth, normal, facet, None)
    want = np.stack([np.frombuffer(oracle.color_encode(v / np.float32(spp)), np.uint8)
                     for v in accum.reshape(-1, 3)]).reshape(h, w, 4)
    assert np.array_equal(got, want)


def test_zero_samples_give_opaque_black(oracle):
    depth, normal, facet, _ = pin_guides(oracle, 8, 6)
    rgba = oracle.denoise_and_tonemap_frame(np.ones((6, 8, 3), np.float32), 0, depth, normal, facet)
    assert np.all(rgba[..., :3] == 0) and np.all(rgba[..., 3] == 255)


def test_tonemap_edge_values(oracle):
    """Non-finite or non-positive XYZ maps to opaque black; every channel stays in
    0..=255 for far out-of-gamut and very bright input (space.rs:226-232)."""
    for v in ([np.nan, 1.0, 1.0], [np.inf, 0.0, 0.0], [0.0, 0.0, 0.0], [-1.0, -1.0, -1.0], [1e-7, 1e-7, 1e-7]):
        assert oracle.color_encode(v) == bytes([0, 0, 0, 255])
    for space in TONEMAP_PINS:
        for v in ([1e6, 1e6, 1e6], [5.0, 0.1, 0.0], [0.0, 3.0, 0.0], [0.0, 0.0, 9.0], [2.0, -1.0, 0.5]):
            out = oracle.color_encode(v, space)
            assert out[3] == 255
    assert oracle.tonemap_to_rgba(np.zeros((0, 3), np.float32)).shape == (0, 4)


def test_signature_zero_without_index_and_guides_unchanged(oracle):
    d0, n0, f0, s0 = pin_guides(oracle)
    assert np.all(s0 == 0)
    d1, n1, f1, s1 = pin_guides(oracle, n_d=2.417)
    assert np.array_equal(f0, f1) and np.array_equal(n0, n1)
    assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))


def test_signature_zero_exactly_on_misses(oracle):
    _, _, facet, sig = pin_guides(oracle, 48, 32, n_d=2.417)
    assert (facet == -1).any() and (facet >= 0).any()
    assert np.array_equal(sig == 0, facet < 0)


def test_signature_regions_and_threads(oracle):
    cam = oracle.camera_new(*PIN_POSE)
    planes = oracle.standard_round_brilliant()
    one = oracle.generate_guide_buffers(61, 37, cam, planes, 2.417, threads=1)
    assert len(set(one[3].ravel().tolist())) > 4
    for t in (2, 8):
        multi = oracle.generate_guide_buffers(61, 37, cam, planes, 2.417, threads=t)
        assert np.array_equal(multi[3], one[3])
    diamond = oracle.generate_guide_buffers(64, 48, cam, planes, 2.417)
    glass = oracle.generate_guide_buffers(64, 48, cam, planes, 1.52)
    assert not np.array_equal(diamond[3], glass[3])
    assert np.array_equal(diamond[2], glass[2])


def test_constant_signature_is_identical_to_none(oracle):
    depth, normal, facet, _ = pin_guides(oracle, 61, 47)
    color = irregular_colors(61 * 47, 0x5151).reshape(47, 61, 3) * np.float32(0.25)
    a = oracle.atrous_denoise(color, depth, normal, facet, None, 1)
    b = oracle.atrous_denoise(color, depth, normal, facet, np.full((47, 61), 0xDEAD, np.uint32), 1)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    # A varied signature changes the result, and the thread count does not.
    sig = ((np.arange(61 * 47) % 61) // 6 + (np.arange(61 * 47) // 61) // 5).astype(np.uint32).reshape(47, 61) % 4
    c1 = oracle.atrous_denoise(color, depth, normal, facet, sig, 1, threads=1)
    c8 = oracle.atrous_denoise(color, depth, normal, facet, sig, 1, threads=8)
    assert np.array_equal(c1.view(np.uint32), c8.view(np.uint32))
    assert not np.array_equal(c1, a)


def test_denoise_keeps_background_and_sanitises_non_finite(oracle):
    """A background pixel (facet < 0) is copied through; a non-finite texel reaches no
    neighbour, and as a pixel's own value it is treated as black."""
    depth, normal, facet, _ = pin_guides(oracle, 32, 24)
    color = irregular_colors(32 * 24, 0x77).reshape(24, 32, 3)
    hit = np.argwhere(facet >= 0)
    y, x = hit[len(hit) // 2]
    color[y, x] = [np.nan, 1.0, 1.0]
    out = oracle.atrous_denoise(color, depth, normal, facet, None, 2)
    assert np.all(np.isfinite(out[facet >= 0]))
    bg = facet < 0
    assert np.array_equal(out[bg].view(np.uint32), color[bg].view(np.uint32))
