"""Record batches on the GPU: words, per-record hits and counts equal the
oracle run on the normalised (separator-joined) sequence."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def _batch(rng, n_records, lo, hi, alphabet=b"ACGT", gap=True):
    parts, ranges, pos = [], [], 0
    for _ in range(n_records):
        if gap and rng.random() < 0.3:
            g = int(rng.integers(1, 20))
            parts.append(random_dna(rng, g, b"ACGT"))
            pos += g
        n = int(rng.integers(lo, hi + 1))
        parts.append(random_dna(rng, n, alphabet))
        ranges.append((pos, n))
        pos += n
    return np.concatenate(parts) if parts else np.zeros(0, np.uint8), ranges


@pytest.mark.parametrize("n_records,lo,hi", [(1, 100, 100), (7, 0, 60), (300, 20, 400),
                                              (40, 1000, 30000)])
def test_insert_record_batch(sbf, cuda, oracle_mod, n_records, lo, hi):
    rng = np.random.default_rng(n_records * 13 + hi)
    seq, ranges = _batch(rng, n_records, lo, hi, b"ACGTACGTACGTN")
    bits = 1 << 20
    f = sbf.Filter(bits, **K31)
    rep = f.insert_record_batch(seq, ranges)
    joined, recs = sbf.normalize_record_batch(31, seq, ranges)
    o = oracle_mod.Oracle(**K31)
    w = o.new_words(bits)
    o.insert(w, joined)
    np.testing.assert_array_equal(f.words_host(), w)
    assert rep.records_indexed == n_records
    assert rep.indexed_bases == sum(n for _, n in ranges)
    assert rep.inserted_kmers == sum(r.valid_kmers for r in recs)


@pytest.mark.parametrize("n_records,lo,hi", [(5, 0, 50), (500, 10, 300), (30, 2000, 40000)])
def test_query_record_batch(sbf, cuda, oracle_mod, n_records, lo, hi):
    rng = np.random.default_rng(n_records + lo)
    seq, ranges = _batch(rng, n_records, lo, hi, b"ACGTACGTACGTN")
    bits = 1 << 18
    f = sbf.Filter(bits, **K31)
    ins_seq, ins_ranges = _batch(rng, 20, 100, 5000)
    f.insert_record_batch(ins_seq, ins_ranges)
    # also insert half of the query records so there are positives
    half = ranges[: len(ranges) // 2]
    f.insert_record_batch(seq, half)
    o = oracle_mod.Oracle(**K31)
    w = f.words_host()
    joined, recs = sbf.normalize_record_batch(31, seq, ranges)
    layout, total = sbf.query_layout(31, recs)
    want_hits = o.contains(w, joined)
    assert want_hits.size == total
    got = []
    rep = f.query_record_batch(seq, ranges, consume=got.append)
    assert len(got) == n_records
    pos_total = 0
    for g, lay, (off, n) in zip(got, layout, ranges):
        h = want_hits[lay.hit_offset:lay.hit_offset + lay.hit_count]
        np.testing.assert_array_equal(g["hits"], h)
        assert g["positive_kmers"] == int(h.sum())
        assert g["queried_kmers"] == lay.valid_kmers
        assert g["queried_bases"] == n
        assert g["sequence"] == seq[off:off + n].tobytes()
        pos_total += int(h.sum())
    assert rep.records_queried == n_records
    assert rep.positive_kmers == pos_total
    assert rep.queried_kmers == sum(r.valid_kmers for r in recs)
    # aggregate-only call agrees
    rep2 = f.query_record_batch(seq, ranges)
    assert (rep2.positive_kmers, rep2.queried_kmers) == (rep.positive_kmers, rep.queried_kmers)


def test_device_record_batch_known_answer(sbf, cuda):
    """tests/test_bloom_filter.cu:342-422 of the reference."""
    torch = cuda
    c5 = dict(k=5, s=4, m=3, hashes=4)
    r1, r2 = b"ACGTACGTACGT", b"TTGGAACCTTGG"
    dev = torch.tensor(list(r1 + b"N" + r2), dtype=torch.uint8, device="cuda")
    ranges = [(0, 12), (13, 12)]
    f = sbf.Filter(1 << 14, **c5)
    assert f.insert_record_batch_async(dev, ranges) == 16
    torch.cuda.synchronize()
    assert f.contains_sequence(r1).all() and f.contains_sequence(r2).all()
    g = sbf.Filter(1 << 14, **c5)
    g.insert_sequence(r1)
    g.insert_sequence(r2)
    out = torch.zeros(21, dtype=torch.uint8, device="cuda")
    g.contains_record_batch_async(dev, ranges, out)
    torch.cuda.synchronize()
    assert out.cpu().tolist() == [1] * 8 + [0] * 5 + [1] * 8
    with pytest.raises(sbf.SbfError):
        g.contains_record_batch_async(dev, ranges, out[:20])
    with pytest.raises(sbf.SbfError):
        g.insert_record_batch_async(dev, [(13, 12), (0, 12)])
