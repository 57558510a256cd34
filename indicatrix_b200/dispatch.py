"""Sample-range dispatch and the deterministic merge (include/ix_dispatch.h), plus the
multi-process plumbing that uses them.

The reference's indicatrix-dispatch hands disjoint absolute sample ranges to lanes and
folds their per-pixel sums in ascending first-sample order
(crates/indicatrix-dispatch/src/sample_cursor/mod.rs, merge/mod.rs).  Here a lane is a
rank of a ``torch.distributed`` group (one per GPU, or gloo ranks on CPU): ranks claim
chunks from a cursor shared through the process group's store, trace them, and rank 0
merges every rank's (first_sample, done, sums) in sample order.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Tuple

import numpy as np

from .backend import load_library

_bound = False


def _lib():
    global _bound
    lib = load_library()
    if not _bound:
        P = C.POINTER
        lib.ix_sample_cursor_new.restype = C.c_void_p
        lib.ix_sample_cursor_new.argtypes = [C.c_uint32, C.c_uint32]
        lib.ix_sample_cursor_free.argtypes = [C.c_void_p]
        lib.ix_sample_cursor_claim.argtypes = [C.c_void_p, C.c_uint32, P(C.c_uint32), P(C.c_uint32)]
        lib.ix_sample_cursor_requeue.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        lib.ix_sample_cursor_fully_claimed.argtypes = [C.c_void_p]
        lib.ix_merger_new.restype = C.c_void_p
        lib.ix_merger_new.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64]
        lib.ix_merger_new_shared.restype = C.c_void_p
        lib.ix_merger_new_shared.argtypes = [C.c_uint64, C.c_uint32, C.c_void_p]
        lib.ix_parked_budget_new.restype = C.c_void_p
        lib.ix_parked_budget_new.argtypes = [C.c_uint64]
        lib.ix_parked_budget_free.argtypes = [C.c_void_p]
        lib.ix_parked_budget_used.restype = C.c_uint64
        lib.ix_parked_budget_used.argtypes = [C.c_void_p]
        lib.ix_merger_free.argtypes = [C.c_void_p]
        lib.ix_merger_add.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, P(C.c_double), C.c_uint64,
                                      P(C.c_uint32)]
        lib.ix_merger_frontier.restype = C.c_uint32
        lib.ix_merger_frontier.argtypes = [C.c_void_p]
        lib.ix_merger_total.restype = C.c_uint32
        lib.ix_merger_total.argtypes = [C.c_void_p]
        lib.ix_merger_dropped_pixels.restype = C.c_uint64
        lib.ix_merger_dropped_pixels.argtypes = [C.c_void_p]
        lib.ix_merger_snapshot.restype = C.c_uint32
        lib.ix_merger_snapshot.argtypes = [C.c_void_p, P(C.c_double), C.c_uint64]
        lib.ix_merger_finish.restype = C.c_uint32
        lib.ix_merger_finish.argtypes = [C.c_void_p, P(C.c_double), C.c_uint64]
        _bound = True
    return lib


MERGE_OK, MERGE_WRONG_LENGTH, MERGE_OVERLAP, MERGE_BUDGET = 0, -1, -2, -3


class MergeError(RuntimeError):
    pass


class SampleCursor:
    """SampleCursor (sample_cursor/mod.rs:64): disjoint absolute ranges in order."""

    def __init__(self, start: int, end: int):
        self._lib = _lib()
        self._h = self._lib.ix_sample_cursor_new(start, end)

    def claim(self, want: int) -> Optional[Tuple[int, int]]:
        s, n = C.c_uint32(), C.c_uint32()
        if self._lib.ix_sample_cursor_claim(self._h, want, C.byref(s), C.byref(n)):
            return int(s.value), int(n.value)
        return None

    def requeue(self, start: int, count: int) -> None:
        self._lib.ix_sample_cursor_requeue(self._h, start, count)

    def fully_claimed(self) -> bool:
        return bool(self._lib.ix_sample_cursor_fully_claimed(self._h))

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ix_sample_cursor_free(self._h)
            self._h = None


class ParkedBudget:
    """A byte budget several mergers park against (ParkedBudget, merge/mod.rs:72)."""

    def __init__(self, bytes_: int):
        self._lib = _lib()
        self._h = self._lib.ix_parked_budget_new(bytes_)

    @property
    def used(self) -> int:
        return int(self._lib.ix_parked_budget_used(self._h))

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ix_parked_budget_free(self._h)
            self._h = None


class Merger:
    """Merger (merge/mod.rs:155): left fold of chunk sums in ascending first-sample
    order; chunks ahead of the frontier are parked, charged against an own byte budget
    (``parked_budget_bytes``) or a shared ``ParkedBudget``."""

    def __init__(self, pixels: int, first_sample: int = 0, parked_budget_bytes: int = 0,
                 shared_budget: Optional["ParkedBudget"] = None):
        self._lib = _lib()
        self.pixels = pixels
        self._budget = shared_budget  # kept alive while this merger uses it
        if shared_budget is not None:
            self._h = self._lib.ix_merger_new_shared(pixels, first_sample, shared_budget._h)
        else:
            self._h = self._lib.ix_merger_new(pixels, first_sample, parked_budget_bytes)

    def add(self, first_sample: int, done: int, sums: np.ndarray) -> int:
        s = np.ascontiguousarray(sums, np.float64).reshape(-1)
        total = C.c_uint32()
        rc = self._lib.ix_merger_add(self._h, first_sample, done, s.ctypes.data_as(C.POINTER(C.c_double)),
                                     s.size, C.byref(total))
        if rc != MERGE_OK:
            raise MergeError({MERGE_WRONG_LENGTH: "wrong length", MERGE_OVERLAP: "overlap",
                              MERGE_BUDGET: "parked budget exceeded"}.get(rc, str(rc)))
        return int(total.value)

    @property
    def frontier(self) -> int:
        return int(self._lib.ix_merger_frontier(self._h))

    @property
    def total(self) -> int:
        return int(self._lib.ix_merger_total(self._h))

    @property
    def dropped_pixels(self) -> int:
        return int(self._lib.ix_merger_dropped_pixels(self._h))

    def snapshot(self) -> Tuple[np.ndarray, int]:
        dst = np.zeros(self.pixels * 3)
        n = self._lib.ix_merger_snapshot(self._h, dst.ctypes.data_as(C.POINTER(C.c_double)), dst.size)
        return dst, int(n)

    def finish(self) -> Tuple[np.ndarray, int]:
        dst = np.zeros(self.pixels * 3)
        n = self._lib.ix_merger_finish(self._h, dst.ctypes.data_as(C.POINTER(C.c_double)), dst.size)
        return dst, int(n)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ix_merger_free(self._h)
            self._h = None


def fold_in_order(parts):
    """Merger::add's fold (merge/mod.rs:239) of per-rank sums that are contiguous sample
    ranges in rank order -- rank r traced [r n, (r + 1) n) -- so rank order is ascending
    first-sample order: left to right, each part added into the running sums.  Works on
    numpy arrays and on torch tensors (on the device that holds them)."""
    acc = parts[0].copy() if isinstance(parts[0], np.ndarray) else parts[0].clone()
    for p in parts[1:]:
        acc += p
    return acc


def gather_fold(sums, group=None):
    """The one exchange step of a sharded render: every rank's per-pixel sums (a torch
    tensor, the same shape on every rank) go to rank 0 with one gather over the process
    group (NCCL over NVLink between GPUs, gloo on CPU), and rank 0 folds them in rank
    order with fold_in_order.  Returns the folded sums on rank 0 and None on the others.
    Every rank takes the same collective step."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    parts = [torch.empty_like(sums) for _ in range(world)] if rank == 0 else None
    dist.gather(sums, parts, dst=0, group=group)
    if rank != 0:
        return None
    return fold_in_order(parts)


def store_claim(store, key: str, start: int, end: int, want: int) -> Optional[Tuple[int, int]]:
    """A SampleCursor shared by every rank through a torch.distributed store: the store's
    atomic add hands out disjoint ranges of `want` samples."""
    hi = int(store.add(key, want))
    lo = hi - want
    s = start + lo
    if s >= end:
        return None
    return s, min(want, end - s)


def distributed_accumulate(trace: Callable[[int, int], np.ndarray], pixels: int, start: int, end: int,
                           chunk: int, key: str = "ix_cursor") -> Optional[Tuple[np.ndarray, int]]:
    """Every rank claims chunks of `chunk` samples from [start, end) through the process
    group's store, traces each with ``trace(first_sample, count) -> sums``, and rank 0
    merges all ranks' chunks in ascending first-sample order.  Returns (sums, samples)
    on rank 0, None elsewhere.  Every rank takes the same collective steps."""
    import torch.distributed as dist

    store = dist.distributed_c10d._get_default_store()
    mine: List[Tuple[int, int, np.ndarray]] = []
    while True:
        c = store_claim(store, key, start, end, chunk)
        if c is None:
            break
        mine.append((c[0], c[1], np.ascontiguousarray(trace(c[0], c[1]), np.float64).reshape(-1)))
    gathered: List = [None] * dist.get_world_size()
    dist.all_gather_object(gathered, mine)
    if dist.get_rank() != 0:
        return None
    m = Merger(pixels, start)
    for chunks in gathered:
        for first, done, sums in chunks:
            m.add(first, done, sums)
    return m.finish()


def distributed_accumulate_payloads(trace: Callable[[int, int], np.ndarray], width: int, height: int, start: int,
                                    end: int, chunk: int, encoding: int = 2,
                                    key: str = "ix_payload_cursor") -> Optional[Tuple[np.ndarray, int, int]]:
    """The lanes' wire form of `distributed_accumulate`: every chunk's per-pixel sums go
    over the group as a radiance payload (Vec3 f32, byte-shuffled and LZ4-compressed when
    that is smaller; indicatrix-net radiance/payload.rs), and rank 0 checks each frame's
    sample range against the request -- a frame outside [start, end) or one that would
    take the cumulative count past the range is refused (RadianceError FrameOutsideRange /
    SampleCountOverrun, radiance/mod.rs:109-117) -- then decodes and adds the frames into
    f32 sums in ascending first-sample order with the valid-sample rule.  Returns
    (sums [pixels, 3] f32, samples, dropped pixels) on rank 0, None elsewhere."""
    import torch.distributed as dist

    from .radiance import PayloadDecoder, PayloadEncoder, RadianceError

    store = dist.distributed_c10d._get_default_store()
    enc = PayloadEncoder(encoding)
    mine = []
    while True:
        c = store_claim(store, key, start, end, chunk)
        if c is None:
            break
        sums = np.ascontiguousarray(trace(c[0], c[1]), np.float64).reshape(-1)
        p = enc.encode(sums.astype(np.float32).tobytes())
        mine.append((c[0], c[1], int(p.encoding), p.raw_len, p.bytes))
    gathered: List = [None] * dist.get_world_size()
    dist.all_gather_object(gathered, mine)
    if dist.get_rank() != 0:
        return None
    frames = sorted((f for chunks in gathered for f in chunks), key=lambda f: f[0])
    acc = np.zeros((width * height, 3), np.float32)
    dec = PayloadDecoder()
    cumulative, dropped = 0, 0
    for first, done, encoding_used, raw_len, wire in frames:
        if first < start or first + done > end:
            raise RadianceError(9)
        if cumulative + done > end - start:
            raise RadianceError(10)
        dropped += dec.decode_and_add(encoding_used, raw_len, wire, width, height, acc)
        cumulative += done
    return acc, cumulative, dropped
