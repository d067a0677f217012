"""sbf_record_batch_counts_noalloc (collected last): per-record counts of a
device record batch from the library's static scratch equal the per-record
queried/positive k-mers of sbf_query_record_batch, on two calls in a row."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def _batch(rng, n_records, lo, hi):
    parts, ranges, pos = [], [], 0
    for _ in range(n_records):
        if rng.random() < 0.3:
            g = int(rng.integers(1, 20))
            parts.append(random_dna(rng, g, b"ACGT"))
            pos += g
        n = int(rng.integers(lo, hi + 1))
        parts.append(random_dna(rng, n, b"ACGTACGTACGTN"))
        ranges.append((pos, n))
        pos += n
    return np.concatenate(parts), ranges


@pytest.mark.parametrize("n_records,lo,hi", [(1, 5000, 5000), (400, 0, 300), (25, 1000, 70000)])
def test_counts_match_query_record_batch(sbf, cuda, n_records, lo, hi):
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
    d_seq = torch.from_numpy(joined.copy()).cuda()
    windows = f.kmer_count(joined.size)
    d_hits = torch.zeros(max(windows, 1), dtype=torch.uint8, device="cuda")
    f.contains_record_batch_async(d_seq, dev_ranges, d_hits)
    torch.cuda.synchronize()
    for _ in range(2):
        valid, pos = f.record_batch_counts_noalloc(d_seq, dev_ranges, d_hits)
        np.testing.assert_array_equal(valid, want_valid)
        np.testing.assert_array_equal(pos, want_pos)
    valid, pos = f.record_batch_counts_noalloc(d_seq, dev_ranges)
    np.testing.assert_array_equal(valid, want_valid)
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
