"""Sharded multi-rank insert on CPU ranks (gloo): every rank emits the run
records of its window slice (oracle), routes them to the owners of their
shards with one all-to-all, ORs what it owns, and all-gathers the shard
ranges.  Every rank's filter must equal the oracle's single insert of the
whole input, word for word.  The device kernels of the same steps are checked
against the engine's own insert in tests/test_sharded_gpu.py."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
K31 = dict(k=31, s=28, m=16, hashes=4)
N_SHARDS = 1 << 12


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sequence():
    rng = np.random.default_rng(2024)
    seq = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 300_000)].copy()
    seq[rng.integers(0, seq.size, 40)] = ord("N")
    seq[1000:1200] = seq[5000:5200]  # a repeat
    return seq


def _rank_main(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle

    from cusbf_b200 import sharded

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        seq = _sequence()
        o = Oracle(**K31, threads=1)
        b0, b1 = sharded.byte_slice(seq.size, 31, world, rank)
        shards, masks = o.runs(seq[b0:b1], N_SHARDS)
        rec = sharded.pack_records(torch.from_numpy(shards.astype(np.int64)),
                                   torch.from_numpy(masks.view(np.int64)), torch)
        mine = sharded.route_records(rec, N_SHARDS, None, torch, dist).numpy()
        per = sharded.shards_per_owner(N_SHARDS, world)
        lo, hi = rank * per, min((rank + 1) * per, N_SHARDS)
        assert mine.shape[0] == 0 or (mine[:, 0].min() >= lo and mine[:, 0].max() < hi)
        words = np.zeros(N_SHARDS * 4, np.uint64)
        sharded.apply_records_host(words, mine, lo, hi)
        t = torch.from_numpy(words.view(np.int64))
        sharded.gather_shards(t, N_SHARDS, None, torch, dist)
        q.put((rank, int(shards.size), int(mine.shape[0]), t.numpy().view(np.uint64).copy()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_gloo_ranks_build_the_single_insert_filter(oracle_mod, world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seq = _sequence()
    o = oracle_mod.Oracle(**K31)
    want = np.zeros(N_SHARDS * 4, np.uint64)
    o.insert(want, seq)
    emitted = sum(r[1] for r in res)
    received = sum(r[2] for r in res)
    assert emitted == received > 0
    for _, _, _, words in res:
        np.testing.assert_array_equal(words, want)


def test_slices_cover_every_window_once():
    sys.path.insert(0, ROOT)
    from cusbf_b200 import sharded

    for n_bytes in (0, 30, 31, 32, 1000, 12345):
        for world in (1, 2, 3, 8):
            n_windows = max(0, n_bytes - 30)
            covered = []
            for r in range(world):
                w0, w1 = sharded.window_range(n_windows, world, r)
                b0, b1 = sharded.byte_slice(n_bytes, 31, world, r)
                assert (b1 - b0) == (w1 - w0 + 30 if w1 > w0 else 0)
                covered.extend(range(w0, w1))
            assert covered == list(range(n_windows))


def test_owner_ranges_split_the_shards():
    sys.path.insert(0, ROOT)
    from cusbf_b200 import sharded

    for n_shards in (1, 4, 4096, 1 << 28):
        for world in (1, 2, 3, 8):
            per = sharded.shards_per_owner(n_shards, world)
            sh = np.array([0, n_shards // 2, n_shards - 1], np.int64)
            own = sharded.owner_of(sh, n_shards, world)
            assert own.min() >= 0 and own.max() < world
            assert per * world >= n_shards
