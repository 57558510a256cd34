"""The radiance frame codec (include/ix_radiance.h) on the host, against the oracle's
restatement (oracle/radiance_oracle.py) and the reference's own codec tests
(crates/indicatrix-net/src/radiance/shuffle.rs tests, payload_tests.rs, mod.rs tests):
shuffle golden bytes and round trips over every special f32 pattern, the valid-sample add,
round trips of every encoding, shrink / raw fallback, the bounded-decode checks in the
reference's order (size cap, raw_len, encoding, decompression bound, short output), and
LZ4 block-format conformance both ways with the oracle's decoder and hand-built blocks.
"""
import numpy as np
import pytest

import radiance_oracle as ro
from indicatrix_b200 import radiance as rad
from indicatrix_b200.radiance import PayloadDecoder, PayloadEncoder, PayloadEncoding, RadianceError

SPECIAL_BITS = [0x00000000, 0x80000000, 0x7FC00000, 0x7FC01234, 0xFFC5A5A5, 0x7F800001, 0xFF800001,
                0x7F800000, 0xFF800000, 0x00000001, 0x807FFFFF, 0x3F800000]


def mixed_bits(n: int, seed: int) -> np.ndarray:
    """test_support.rs mixed_bits: xorshift32, every third value a special pattern."""
    s = (seed | 1) & 0xFFFFFFFF
    out = np.zeros(n, np.uint32)
    for i in range(n):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        out[i] = SPECIAL_BITS[(i // 3) % len(SPECIAL_BITS)] if i % 3 == 0 else s
    return out


def smooth_payload(pixels: int) -> bytes:
    """test_support.rs smooth_payload: a gradient with low-bit noise."""
    s = 0x9E3779B9
    vals = np.zeros(pixels * 3, np.uint32)
    for i in range(pixels * 3):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        base = np.float32(1.0) + np.float32(i % 97) / np.float32(97.0)
        vals[i] = int(np.array([base], np.float32).view(np.uint32)[0]) ^ (s & 0xFF)
    return vals.tobytes()


def test_shuffle_groups_bytes_by_plane():
    raw = bytes([0x10, 0x11, 0x12, 0x13, 0x20, 0x21, 0x22, 0x23])
    out = np.zeros(8, np.uint8)
    rad.shuffle_into(raw, out)
    assert out.tobytes() == bytes([0x10, 0x20, 0x11, 0x21, 0x12, 0x22, 0x13, 0x23])


@pytest.mark.parametrize("n,seed", [(0, 1), (1, 2), (3, 3), (12, 4), (997, 5), (3 * 4096, 6)])
def test_shuffle_round_trips_bit_exactly(n, seed):
    raw = mixed_bits(n, seed).tobytes()
    sh = np.zeros(len(raw), np.uint8)
    back = np.zeros(len(raw), np.uint8)
    rad.shuffle_into(raw, sh)
    assert sh.tobytes() == ro.shuffle(raw)
    rad.unshuffle_into(sh, back)
    assert back.tobytes() == raw


def test_shuffle_rejects_a_partial_value():
    with pytest.raises(RadianceError):
        rad.shuffle_into(bytes([1, 2, 3]), np.zeros(3, np.uint8))


def test_add_unshuffled_valid_skips_and_counts_invalid_pixels():
    pixels = np.array([[1, 2, 3], [np.nan, 1, 1], [1, np.inf, 1], [1, 1, -0.5], [0.0, -0.0, 4.0]], np.float32)
    raw = pixels.tobytes()
    acc = np.ones((5, 3), np.float32)
    dropped = PayloadDecoder().decode_and_add(PayloadEncoding.RAW, len(raw), raw, 5, 1, acc)
    assert dropped == 3
    assert np.array_equal(acc, np.array([[2, 3, 4], [1, 1, 1], [1, 1, 1], [1, 1, 1], [1, 1, 5]], np.float32))
    assert not rad.is_valid_sample([1, 1, -0.5]) and rad.is_valid_sample([0.0, -0.0, 4.0])


@pytest.mark.parametrize("encoding", [PayloadEncoding.RAW, PayloadEncoding.SHUFFLE_LZ4, PayloadEncoding.SHUFFLE_ZSTD])
def test_every_encoding_round_trips_bit_exactly(encoding):
    for (w, h), seed in [((1, 1), 3), ((7, 5), 4), ((64, 48), 5)]:
        raw = mixed_bits(w * h * 3, seed).tobytes()
        for payload_raw in (raw, smooth_payload(w * h)):
            p = PayloadEncoder(encoding).encode(payload_raw)
            assert p.raw_len == len(payload_raw)
            if encoding == PayloadEncoding.SHUFFLE_ZSTD:
                assert p.encoding == PayloadEncoding.RAW  # not supported here: Raw
            out = PayloadDecoder().decode_to_vec(p.encoding, p.raw_len, p.bytes, w, h)
            assert out.tobytes() == payload_raw


def test_decode_and_add_is_bit_identical_to_the_raw_path():
    w, h = 33, 21
    delta = np.frombuffer(mixed_bits(w * h * 3, 9).tobytes(), np.float32).reshape(-1, 3)
    start = np.abs(np.frombuffer(mixed_bits(w * h * 3, 10).tobytes(), np.float32)).reshape(-1, 3).copy()
    start[~np.isfinite(start)] = 1.0
    want = start.copy()
    dropped_want = ro.add_valid(want, delta)
    for enc in (PayloadEncoding.RAW, PayloadEncoding.SHUFFLE_LZ4):
        p = PayloadEncoder(enc).encode(delta.tobytes())
        acc = start.copy()
        dropped = PayloadDecoder().decode_and_add(p.encoding, p.raw_len, p.bytes, w, h, acc)
        assert dropped == dropped_want
        assert np.array_equal(acc.view(np.uint32), want.view(np.uint32))


def test_compressible_payloads_shrink_and_incompressible_ones_go_raw():
    smooth = smooth_payload(4096)
    rng = np.random.default_rng(0x12345678)
    noise = rng.integers(0, 256, len(smooth), dtype=np.uint8).tobytes()
    enc = PayloadEncoder(PayloadEncoding.SHUFFLE_LZ4)
    p = enc.encode(smooth)
    assert p.encoding == PayloadEncoding.SHUFFLE_LZ4 and len(p.bytes) < len(smooth)
    p = enc.encode(noise)
    assert p.encoding == PayloadEncoding.RAW and p.bytes == noise


def test_lying_raw_len_and_size_caps():
    dec = PayloadDecoder()
    raw = smooth_payload(4)
    acc = np.zeros((4, 3), np.float32)
    with pytest.raises(RadianceError) as e:
        dec.decode_and_add(PayloadEncoding.RAW, len(raw) + 12, raw, 2, 2, acc)
    assert e.value.name == "RawLenMismatch"
    # width * height * 12 over MAX_FRAME_LEN is refused before anything else.
    big_w = rad.MAX_FRAME_LEN // 12 + 1
    with pytest.raises(RadianceError) as e:
        dec.decode_to_vec(PayloadEncoding.SHUFFLE_LZ4, 0, b"", big_w, 1)
    assert e.value.name == "TooLarge"
    # Exactly at the cap: the raw_len check is reached (and fails on a lying header).
    w = rad.MAX_FRAME_LEN // 12 // 4096
    with pytest.raises(RadianceError) as e:
        dec.decode_to_vec(PayloadEncoding.SHUFFLE_LZ4, 12, b"\x00", w, 4096)
    assert e.value.name == "RawLenMismatch"
    with pytest.raises(RadianceError) as e:
        dec.decode_to_vec(PayloadEncoding.SHUFFLE_LZ4, 12, b"\x00", w, 4097)
    assert e.value.name == "TooLarge"
    with pytest.raises(RadianceError) as e:
        dec.decode_to_vec(PayloadEncoding.RAW, 48, raw[:47], 2, 2)
    assert e.value.name == "LengthMismatch"


def test_an_expansion_bomb_is_rejected():
    w, h = 64, 64
    raw_len = w * h * 12
    bomb = PayloadEncoder(PayloadEncoding.SHUFFLE_LZ4).encode(bytes(raw_len * 64))
    assert bomb.encoding == PayloadEncoding.SHUFFLE_LZ4 and len(bomb.bytes) < raw_len
    with pytest.raises(RadianceError) as e:
        PayloadDecoder().decode_to_vec(bomb.encoding, raw_len, bomb.bytes, w, h)
    assert e.value.name == "DecompressFailed"


def test_a_short_payload_is_rejected():
    w, h = 16, 16
    half = PayloadEncoder(PayloadEncoding.SHUFFLE_LZ4).encode(smooth_payload(w * h // 2))
    assert half.encoding == PayloadEncoding.SHUFFLE_LZ4
    with pytest.raises(RadianceError) as e:
        PayloadDecoder().decode_to_vec(half.encoding, w * h * 12, half.bytes, w, h)
    assert e.value.name in ("ShortOutput", "DecompressFailed")


def test_corrupt_and_unsupported_payloads_are_rejected():
    with pytest.raises(RadianceError) as e:
        PayloadDecoder().decode_to_vec(PayloadEncoding.SHUFFLE_LZ4, 48, bytes([0xFF] * 64), 2, 2)
    assert e.value.name == "DecompressFailed"
    with pytest.raises(RadianceError) as e:
        PayloadDecoder().decode_to_vec(PayloadEncoding.SHUFFLE_ZSTD, 48, bytes(10), 2, 2)
    assert e.value.name == "UnsupportedEncoding"
    # zero-area payloads decode to nothing, whatever the encoding claims.
    assert PayloadDecoder().decode_to_vec(PayloadEncoding.SHUFFLE_LZ4, 0, b"", 0, 5).shape == (0, 3)
    with pytest.raises(RadianceError):
        PayloadDecoder().decode_and_add(PayloadEncoding.RAW, 48, bytes(48), 2, 2, np.zeros((3, 3), np.float32))


def test_lz4_blocks_conform_to_the_format_both_ways():
    """Our blocks decode with the oracle's format decoder; hand-built blocks (overlapping
    matches, literal and match runs needing extension bytes) decode with ours."""
    rng = np.random.default_rng(5)
    for raw in (smooth_payload(300), bytes(1000), rng.integers(0, 4, 4000, dtype=np.uint8).tobytes(),
                mixed_bits(999, 7).tobytes()):
        p = PayloadEncoder(PayloadEncoding.SHUFFLE_LZ4).encode(raw)
        if p.encoding == PayloadEncoding.SHUFFLE_LZ4:
            assert ro.unshuffle(ro.lz4_block_decode(p.bytes, len(raw))) == raw
    # Hand-built: 300 literal bytes, an RLE match of 700 at offset 1, a match of 20 at
    # offset 13, then 40 literals -> 1060 raw bytes (a multiple of 12: 88 pixels + 4 ...).
    lit = rng.integers(0, 256, 300, dtype=np.uint8).tobytes()
    tail = rng.integers(0, 256, 40, dtype=np.uint8).tobytes()
    block = (ro.lz4_sequence(lit, 1, 700) + ro.lz4_sequence(b"", 13, 20) +
             ro.lz4_sequence(tail, last=True))
    want = ro.lz4_block_decode(block, 1060)
    assert len(want) == 1060
    pix = 1056 // 12
    block2 = ro.lz4_sequence(lit, 1, 700) + ro.lz4_sequence(b"", 13, 16) + ro.lz4_sequence(tail, last=True)
    want2 = ro.lz4_block_decode(block2, 1056)
    got = PayloadDecoder().decode_to_vec(PayloadEncoding.SHUFFLE_LZ4, 1056, block2, pix, 1)
    assert got.tobytes() == ro.unshuffle(want2)
    # A block whose match reaches back before the start is corrupt.
    bad = ro.lz4_sequence(b"abcd", 9, 8) + ro.lz4_sequence(b"xyzxy", last=True)
    with pytest.raises(ro.Lz4Error):
        ro.lz4_block_decode(bad, 64)
    with pytest.raises(RadianceError) as e:
        PayloadDecoder().decode_to_vec(PayloadEncoding.SHUFFLE_LZ4, 12, bad, 1, 1)
    assert e.value.name == "DecompressFailed"


def test_device_forms_decline_without_a_device():
    from indicatrix_b200.backend import GpuBackend

    with pytest.raises(RadianceError) as e:
        rad.decode_and_add_device(GpuBackend.disabled(), PayloadEncoding.RAW, 12, bytes(12), 1, 1, 0)
    assert e.value.name == "Declined"
    with pytest.raises(RadianceError) as e:
        rad.encode_device(GpuBackend.disabled(), PayloadEncoding.RAW, 0, 1, 1)
    assert e.value.name == "Declined"
