"""TEST INFRASTRUCTURE ONLY: a Python restatement of the radiance frame codec's byte work
(crates/indicatrix-net/src/radiance/shuffle.rs, payload.rs) and of the LZ4 block format
the reference links (lz4_flex 0.14.0, not vendored: restated from the published block
format -- token, literal run, little-endian 16-bit offset, match run of length >= 4,
literal-only last sequence).  The tests use it as the checker of the library's codec;
nothing in ``indicatrix_b200`` imports it.  Pure Python: small inputs only.
"""
from __future__ import annotations

import numpy as np


def shuffle(raw: bytes) -> bytes:
    """shuffle_into (shuffle.rs:35): all byte 0s, then all byte 1s, 2s, 3s."""
    a = np.frombuffer(raw, np.uint8)
    assert a.size % 4 == 0
    return a.reshape(-1, 4).T.copy().tobytes()


def unshuffle(planes: bytes) -> bytes:
    """unshuffle_into (shuffle.rs:60)."""
    a = np.frombuffer(planes, np.uint8)
    assert a.size % 4 == 0
    return a.reshape(4, -1).T.copy().tobytes()


def valid_sample(v: np.ndarray) -> bool:
    """is_valid_sample (shuffle.rs:23)."""
    return bool(np.all(np.isfinite(v)) and np.all(v >= 0))


def add_valid(acc: np.ndarray, values: np.ndarray) -> int:
    """add_unshuffled_valid (shuffle.rs:128) on unshuffled values: returns dropped."""
    dropped = 0
    for p in range(acc.shape[0]):
        v = values[p]
        if valid_sample(v):
            acc[p] = (acc[p] + v).astype(np.float32)
        else:
            dropped += 1
    return dropped


class Lz4Error(Exception):
    pass


def lz4_block_decode(block: bytes, capacity: int) -> bytes:
    """Decode one LZ4 block into at most `capacity` bytes (raises Lz4Error otherwise)."""
    out = bytearray()
    i, n = 0, len(block)
    while True:
        if i >= n:
            raise Lz4Error("truncated")
        token = block[i]
        i += 1
        lit = token >> 4
        if lit == 15:
            while True:
                if i >= n:
                    raise Lz4Error("truncated literal length")
                b = block[i]
                i += 1
                lit += b
                if b != 255:
                    break
        if lit > n - i or len(out) + lit > capacity:
            raise Lz4Error("literal run past the end")
        out += block[i:i + lit]
        i += lit
        if i == n:
            return bytes(out)
        if n - i < 2:
            raise Lz4Error("truncated offset")
        off = block[i] | (block[i + 1] << 8)
        i += 2
        if off == 0 or off > len(out):
            raise Lz4Error("bad offset")
        ml = (token & 15) + 4
        if token & 15 == 15:
            while True:
                if i >= n:
                    raise Lz4Error("truncated match length")
                b = block[i]
                i += 1
                ml += b
                if b != 255:
                    break
        if len(out) + ml > capacity:
            raise Lz4Error("match past the end")
        start = len(out) - off
        for k in range(ml):
            out.append(out[start + k])


def lz4_sequence(literals: bytes, offset: int = 0, match_len: int = 0, last: bool = False) -> bytes:
    """One sequence of the block format, for building test blocks by hand."""
    lit = len(literals)
    ml = 0 if last else match_len - 4
    out = bytearray([(min(lit, 15) << 4) | (0 if last else min(ml, 15))])
    if lit >= 15:
        r = lit - 15
        while r >= 255:
            out.append(255)
            r -= 255
        out.append(r)
    out += literals
    if not last:
        out += bytes([offset & 0xFF, offset >> 8])
        if ml >= 15:
            r = ml - 15
            while r >= 255:
                out.append(255)
                r -= 255
            out.append(r)
    return bytes(out)
