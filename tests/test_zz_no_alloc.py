"""sbf_record_batch_counts_noalloc (collected last): per-record counts of a
device record batch, computed from the library's static scratch for callers
that cannot allocate device memory at call time (a serving loop whose memory
is reserved at start-up, an allocator hook).

The counts must equal, on two calls in a row:
  * the per-record queried/positive k-mers of sbf_query_record_batch (the
    entry point that allocates);
  * an independent restatement: valid windows by the reference's rule (all K
    bytes A/C/G/T in any case, normalized_record_batch.hpp:88-110) and the
    positives of each record's windows in the oracle's query bytes over the
    same joined batch and filter words.
Batches mix upper and lower case with non-ACGT bytes."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)
K = 31


def _record_bytes(rng, n):
    """n bases in mixed case with non-ACGT bytes (N, n, R, '-') at about 1%."""
    seq = random_dna(rng, n, b"ACGTacgt")
    bad = np.flatnonzero(rng.random(n) < 0.01)
    seq[bad] = np.frombuffer(b"NnR-", np.uint8)[rng.integers(0, 4, bad.size)]
    return seq


def _batch(rng, n_records, lo, hi):
    parts, ranges, pos = [], [], 0
    for _ in range(n_records):
        if rng.random() < 0.3:
            g = int(rng.integers(1, 20))
            parts.append(random_dna(rng, g, b"ACGT"))
            pos += g
        n = int(rng.integers(lo, hi + 1))
        parts.append(_record_bytes(rng, n))
        ranges.append((pos, n))
        pos += n
    return np.concatenate(parts), ranges


def _valid_windows(rec: np.ndarray) -> int:
    """Windows of `rec` whose K bytes are all A/C/G/T, any case
    (valid_record_kmer_count, normalized_record_batch.hpp:88-110)."""
    if rec.size < K:
        return 0
    up = rec & 0xDF
    ok = (up == ord("A")) | (up == ord("C")) | (up == ord("G")) | (up == ord("T"))
    c = np.concatenate([[0], np.cumsum(~ok, dtype=np.int64)])
    return int(np.count_nonzero(c[K:] - c[:-K] == 0))


@pytest.mark.parametrize("n_records,lo,hi", [(1, 5000, 5000), (400, 0, 300), (25, 1000, 70000)])
def test_counts_match_query_record_batch(sbf, cuda, oracle_mod, n_records, lo, hi):
    torch = cuda
    rng = np.random.default_rng(7 * n_records + hi)
    seq, ranges = _batch(rng, n_records, lo, hi)
    f = sbf.Filter(1 << 20, **K31)
    f.insert_record_batch(seq, ranges[::2])
    got = []
    rep = f.query_record_batch(seq, ranges, consume=got.append)
    want_valid = np.array([g["queried_kmers"] for g in got], np.uint64)
    want_pos = np.array([g["positive_kmers"] for g in got], np.uint64)
    assert int(want_pos.sum()) == rep.positive_kmers

    joined, recs = sbf.normalize_record_batch(31, seq, ranges)
    layout, _ = sbf.query_layout(31, recs)
    dev_ranges = [(r.hit_offset, r.size) for r in layout]
    for (a, n), (off, size) in zip(ranges, dev_ranges):
        assert joined[off:off + size].tobytes() == seq[a:a + n].tobytes()

    # Independent expectation: the reference's valid-window rule per record,
    # and positives from the oracle's query bytes of the joined batch.
    ref_valid = np.array([_valid_windows(joined[o:o + n]) for o, n in dev_ranges], np.uint64)
    ref_hits = oracle_mod.Oracle(**K31).contains(f.words_host(), joined)
    ref_pos = np.array([int(ref_hits[o:o + max(0, n - K + 1)].sum()) for o, n in dev_ranges],
                       np.uint64)
    np.testing.assert_array_equal(want_valid, ref_valid)
    np.testing.assert_array_equal(want_pos, ref_pos)

    d_seq = torch.from_numpy(joined.copy()).cuda()
    windows = f.kmer_count(joined.size)
    d_hits = torch.zeros(max(windows, 1), dtype=torch.uint8, device="cuda")
    f.contains_record_batch_async(d_seq, dev_ranges, d_hits)
    torch.cuda.synchronize()
    for _ in range(2):
        valid, pos = f.record_batch_counts_noalloc(d_seq, dev_ranges, d_hits)
        np.testing.assert_array_equal(valid, want_valid)
        np.testing.assert_array_equal(pos, want_pos)
        np.testing.assert_array_equal(valid, ref_valid)
        np.testing.assert_array_equal(pos, ref_pos)
    valid, pos = f.record_batch_counts_noalloc(d_seq, dev_ranges)
    np.testing.assert_array_equal(valid, ref_valid)
    assert not pos.any()


def test_counts_reject_oversized_batch(sbf, cuda):
    torch = cuda
    f = sbf.Filter(1 << 16, **K31)
    n = 262144 + 1
    d_seq = torch.zeros(n, dtype=torch.uint8, device="cuda")
    ranges = np.stack([np.arange(n, dtype=np.uint64), np.ones(n, np.uint64)], axis=1)
    with pytest.raises(sbf.SbfError, match="262144-record limit"):
        f.record_batch_counts_noalloc(d_seq, ranges)
    valid, pos = f.record_batch_counts_noalloc(d_seq, ranges[:262144])
    assert not valid.any() and not pos.any()
