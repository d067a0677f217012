"""Device steps of the sharded multi-rank insert on one GPU: W ranks are
emulated in one process (each rank's window slice emits its run records with
sbf_emit_runs_async, the records are routed to the owners of their shards,
and each owner ORs its records with sbf_apply_runs_async into its shard range
of one filter).  The filter must equal the engine's single insert of the
whole input word for word, and the emitted records must cover the shards of
the oracle's runs of each slice."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


@pytest.mark.parametrize("world,n,bits", [(1, 50_000, 1 << 20), (2, 1_000_000, 1 << 24),
                                          (3, 777_777, 1 << 22), (8, 3_000_000, 1 << 26)])
def test_emulated_ranks_build_the_single_insert_filter(sbf, cuda, oracle_mod, world, n, bits):
    torch = cuda
    from cusbf_b200 import sharded

    rng = np.random.default_rng(world * 1000 + n)
    seq = random_dna(rng, n, b"ACGTACGTACGTACGTacgtN")
    d_seq = torch.from_numpy(seq).cuda()
    want = sbf.Filter(bits, **K31)
    want.insert_sequence_async(d_seq)
    up = seq & 0xDF
    ok = (up == ord("A")) | (up == ord("C")) | (up == ord("G")) | (up == ord("T"))
    c = np.concatenate([[0], np.cumsum(~ok, dtype=np.int64)])
    valid_all = int(np.count_nonzero(c[31:] - c[:-31] == 0))
    f = sbf.Filter(bits, **K31)
    ns = f.num_shards()
    per = sharded.shards_per_owner(ns, world)
    buckets = [[] for _ in range(world)]
    emitted = 0
    for r in range(world):
        b0, b1 = sharded.byte_slice(n, 31, world, r)
        shards, masks, valid = f.emit_runs(d_seq[b0:b1])
        emitted += valid
        if r == 0:
            # Runs that cross a 32-window strip are emitted once per strip, so
            # the records cover the oracle's runs' shards exactly.
            o_sh, _ = oracle_mod.Oracle(**K31).runs(seq[b0:b1], ns)
            np.testing.assert_array_equal(np.unique(shards.cpu().numpy().astype(np.uint32)),
                                          np.unique(o_sh))
            assert shards.numel() >= o_sh.size
        rec = sharded.pack_records(shards, masks, torch)
        owner = sharded.owner_of(rec[:, 0], ns, world)
        for o in range(world):
            buckets[o].append(rec[owner == o])
    assert emitted == valid_all
    for o in range(world):
        mine = torch.cat(buckets[o])
        f.apply_runs(mine[:, 0].to(torch.int32).contiguous(), mine[:, 1:].contiguous(),
                     o * per, min((o + 1) * per, ns))
    f.synchronize()
    assert torch.equal(f.words(), want.words())


def test_misrouted_record_is_reported(sbf, cuda):
    torch = cuda
    f = sbf.Filter(1 << 20, **K31)  # 4096 shards; this rank owns [0, 256)
    shards = torch.tensor([5, 300], dtype=torch.int32, device="cuda")
    masks = torch.ones((2, 4), dtype=torch.int64, device="cuda")
    f.apply_runs(shards, masks, 0, 256)
    with pytest.raises(sbf.SbfError, match="shard range"):
        f.synchronize()
    f.synchronize()  # the error word was cleared
    w = f.words().view(torch.int64).view(-1, 4)
    assert int(w[5].count_nonzero()) == 4 and int(w[300].count_nonzero()) == 0
