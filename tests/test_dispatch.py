"""Sample-range dispatch and deterministic merge (include/ix_dispatch.h) on the CPU,
including a 2-rank gloo run of the multi-process path.

Modelled on the reference's dispatch tests (crates/indicatrix-dispatch/src/merge,
pool/tests/fake.rs): lanes produce deterministic per-pixel sums, and the merged result
must not depend on which lane traced which chunk or in which order chunks arrive.
"""
import os
import pickle
import socket
import tempfile

import numpy as np
import pytest

from indicatrix_b200.dispatch import MergeError, Merger, SampleCursor


def test_sample_cursor_hands_out_disjoint_ranges_and_requeues():
    c = SampleCursor(10, 33)
    got = []
    while True:
        r = c.claim(5)
        if r is None:
            break
        got.append(r)
    assert got == [(10, 5), (15, 5), (20, 5), (25, 5), (30, 3)]
    assert c.fully_claimed()
    c.requeue(20, 5)
    assert not c.fully_claimed()
    assert c.claim(3) == (20, 3) and c.claim(3) == (23, 2) and c.claim(3) is None


def fake_chunk(pixels, first, done, salt=0):
    """A lane's chunk sum: a deterministic function of (pixel, sample), small integers
    plus a non-dyadic part so the fold order shows in the bits."""
    s = np.arange(first, first + done, dtype=np.float64)
    p = np.arange(pixels, dtype=np.float64)[:, None]
    v = (p * 0.1 + s[None, :] * 0.3 + salt) % 7.0 + 0.013
    return np.repeat(v.sum(axis=1)[:, None], 3, axis=1) * np.array([1.0, 1.1, 0.9])


def test_merger_fold_is_order_independent_and_exact():
    pixels = 37
    chunks = [(0, 4), (4, 7), (11, 1), (12, 9), (21, 3)]
    sums = {c: fake_chunk(pixels, *c) for c in chunks}
    ref = Merger(pixels, 0)
    for c in chunks:
        ref.add(c[0], c[1], sums[c])
    want, n = ref.finish()
    assert n == 24
    rng = np.random.default_rng(3)
    for _ in range(6):
        order = list(rng.permutation(len(chunks)))
        m = Merger(pixels, 0)
        for i in order:
            m.add(chunks[i][0], chunks[i][1], sums[chunks[i]])
        got, n2 = m.finish()
        assert n2 == 24 and np.array_equal(got.view(np.uint64), want.view(np.uint64))
    # the fold is ((0 + a) + b) + ... in sample order
    fold = np.zeros((pixels, 3))
    for c in chunks:
        fold = fold + sums[c]
    assert np.array_equal(want.reshape(pixels, 3), fold)


def test_merger_rejects_overlaps_and_bad_lengths_and_drops_invalid_pixels():
    m = Merger(4, 10)
    m.add(12, 2, np.ones((4, 3)))
    assert m.frontier == 10 and m.total == 2
    with pytest.raises(MergeError):
        m.add(13, 1, np.ones((4, 3)))
    with pytest.raises(MergeError):
        m.add(10, 1, np.ones((3, 3)))
    bad = np.ones((4, 3))
    bad[1, 2] = np.nan
    bad[3, 0] = -1.0
    m.add(10, 2, bad)
    assert m.frontier == 14 and m.dropped_pixels == 2
    snap, n = m.snapshot()
    out, n2 = m.finish()
    assert n == n2 == 4 and np.array_equal(snap, out)
    assert out.reshape(4, 3)[1].tolist() == [1.0, 1.0, 1.0] and out.reshape(4, 3)[0].tolist() == [2.0] * 3


def test_merger_parked_budget_refuses_instead_of_growing():
    m = Merger(2, 0, parked_budget_bytes=2 * 3 * 8)  # room for one parked chunk
    m.add(5, 1, np.ones((2, 3)))
    with pytest.raises(MergeError):
        m.add(7, 1, np.ones((2, 3)))
    m.add(0, 5, np.ones((2, 3)))  # folds itself and the parked chunk
    assert m.frontier == 6


def test_mergers_share_one_parked_budget():
    """Merger::with_parked_budget (merge/mod.rs:190) with one budget shared by two mergers,
    as merge/tests.rs:140-230 exercises it: a chunk that must park past the shared cap is
    refused and not counted; filling the gap at the frontier folds the backlog and releases
    its charge; finishing and freeing release exactly what is still parked, once."""
    from indicatrix_b200.dispatch import ParkedBudget

    def chunk(v):
        return np.full(2 * 3, v)

    budget = ParkedBudget(2 * 2 * 3 * 8)  # two 2-pixel chunks of f64 sums
    a = Merger(2, 0, shared_budget=budget)
    b = Merger(2, 0, shared_budget=budget)
    assert a.add(2, 1, chunk(1.0)) == 1 and budget.used == 48
    assert b.add(2, 1, chunk(1.0)) == 1 and budget.used == 96
    with pytest.raises(MergeError):
        b.add(4, 1, chunk(1.0))  # a third parked chunk: over the shared cap
    assert b.total == 1
    assert a.add(0, 2, chunk(1.0)) == 3 and budget.used == 48  # a's backlog folds
    assert b.add(4, 1, chunk(1.0)) == 2 and budget.used == 96  # room again
    sums, n = b.finish()
    assert n == 2 and budget.used == 0  # b's two parked chunks released once (a has none)
    del b
    assert budget.used == 0
    assert a.add(5, 1, chunk(2.0)) == 4 and budget.used == 48  # parks past a's frontier 3
    del a  # freed with that chunk still parked: its charge returns
    assert budget.used == 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_path):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import datetime

    import torch.distributed as dist

    import ix_oracle
    from indicatrix_b200 import workloads
    from indicatrix_b200.dispatch import distributed_accumulate

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    fs = workloads.round_brilliant_frame(8, 6)
    sc = fs.to_abi()

    def trace(first, count):  # a CPU lane: the oracle traces the chunk's samples
        _, s64, _ = ix_oracle.trace_frame(sc, first, count, threads=1)
        return s64

    res = distributed_accumulate(trace, 48, 0, 23, 5)
    if rank == 0:
        with open(out_path, "wb") as f:
            pickle.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sample_sharding_merges_deterministically(oracle):
    """2 gloo ranks claim 5-sample chunks of [0, 23) through the store, trace them on the
    CPU, and rank 0 folds every chunk in sample order: the result equals a single
    process folding the same partition, bit for bit."""
    import torch.multiprocessing as mp

    from indicatrix_b200 import workloads

    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "res.pkl")
        mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        with open(out, "rb") as f:
            sums, n = pickle.load(f)
    assert n == 23
    fs = workloads.round_brilliant_frame(8, 6)
    sc = fs.to_abi()
    want = np.zeros(48 * 3)
    for first in range(0, 23, 5):
        _, s64, _ = oracle.trace_frame(sc, first, min(5, 23 - first), threads=1)
        want = want + s64.reshape(-1)
    assert np.array_equal(sums.view(np.uint64), want.view(np.uint64))


def _rank_payload_main(rank, world, port, out_path):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import datetime

    import torch.distributed as dist

    import ix_oracle
    from indicatrix_b200 import workloads
    from indicatrix_b200.dispatch import distributed_accumulate_payloads

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    fs = workloads.round_brilliant_frame(8, 6)
    sc = fs.to_abi()

    def trace(first, count):
        _, s64, _ = ix_oracle.trace_frame(sc, first, count, threads=1)
        return s64

    res = distributed_accumulate_payloads(trace, 8, 6, 0, 23, 5)
    if rank == 0:
        with open(out_path, "wb") as f:
            pickle.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_lanes_exchange_radiance_payloads(oracle):
    """The wire form: 2 gloo ranks send their chunks as radiance payloads (f32 Vec3,
    shuffled + LZ4 where smaller) and rank 0 decodes and adds them in sample order: the
    f32 sums equal a single process adding the same chunks' f32 frames in that order."""
    import torch.multiprocessing as mp

    from indicatrix_b200 import workloads

    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "res.pkl")
        mp.start_processes(_rank_payload_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        with open(out, "rb") as f:
            acc, n, dropped = pickle.load(f)
    assert n == 23 and dropped == 0
    fs = workloads.round_brilliant_frame(8, 6)  # kept alive: the scene points into its planes
    sc = fs.to_abi()
    want = np.zeros((48, 3), np.float32)
    for first in range(0, 23, 5):
        _, s64, _ = oracle.trace_frame(sc, first, min(5, 23 - first), threads=1)
        want = (want + s64.reshape(-1, 3).astype(np.float32)).astype(np.float32)
    assert want.sum() > 0
    assert np.array_equal(acc.view(np.uint32), want.view(np.uint32))


def _rank_gather_main(rank, world, port, out_path):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import datetime

    import torch
    import torch.distributed as dist

    import ix_oracle
    from indicatrix_b200 import workloads
    from indicatrix_b200.dispatch import gather_fold

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    # Two jobs of different spp, back to back in one buffer, as a batch plan lays them out:
    # rank r traces samples [r spp_j, (r + 1) spp_j) of job j.
    jobs = [(workloads.round_brilliant_frame(6, 5), 4), (workloads.round_brilliant_frame(4, 4), 7)]
    parts = []
    for fs, spp in jobs:
        _, s64, _ = ix_oracle.trace_frame(fs.to_abi(), rank * spp, spp, threads=1)
        parts.append(s64.reshape(-1))
    mine = torch.from_numpy(np.concatenate(parts))
    folded = gather_fold(mine)
    if rank == 0:
        with open(out_path, "wb") as f:
            pickle.dump(folded.numpy(), f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_gather_fold_equals_the_merger(oracle):
    """The batch path's exchange step (bench.py under torchrun): each rank's per-pixel sums
    of every job go to rank 0 in one gather and are folded in rank order; the result
    equals Merger::add folding each job's two sample ranges in first-sample order, bit
    for bit."""
    import torch.multiprocessing as mp

    from indicatrix_b200 import workloads
    from indicatrix_b200.dispatch import Merger

    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "res.pkl")
        mp.start_processes(_rank_gather_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        with open(out, "rb") as f:
            got = pickle.load(f)
    want = []
    for (w, h), spp in (((6, 5), 4), ((4, 4), 7)):
        fs = workloads.round_brilliant_frame(w, h)
        m = Merger(w * h, 0)
        for r in (1, 0):  # arrival order does not matter: the merger parks rank 1's chunk
            _, s64, _ = oracle.trace_frame(fs.to_abi(), r * spp, spp, threads=1)
            m.add(r * spp, spp, s64.reshape(-1))
        sums, n = m.finish()
        assert n == 2 * spp
        want.append(sums)
    want = np.concatenate(want)
    assert want.sum() > 0
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
