"""Ragged batches (sbf_ragged_*): one persistent launch over records in
place equals one plain insert / query per record, checked against the oracle
run record by record, through the host pipeline (any chunking, stages, graph
replay) and the device-resident entry points."""
import os

import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def _batch(rng, n_records, lo, hi, gaps=True, alphabet=b"ACGTACGTACGTACGTN"):
    parts, ranges, pos = [], [], 0
    for _ in range(n_records):
        if gaps and rng.random() < 0.3:
            g = int(rng.integers(1, 40))
            parts.append(random_dna(rng, g, b"ACGT"))
            pos += g
        n = int(rng.integers(lo, hi + 1))
        parts.append(random_dna(rng, n, alphabet))
        ranges.append((pos, n))
        pos += n
    if gaps:
        parts.append(random_dna(rng, 17, b"ACGT"))
    seq = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
    return seq, ranges


def _oracle_words(oracle_mod, bits, seq, ranges, cfg=K31):
    o = oracle_mod.Oracle(**cfg)
    w = o.new_words(bits)
    for off, n in ranges:
        o.insert(w, seq[off:off + n])
    return o, w


TUNINGS = [None,
           dict(chunk_bytes=4096, stages=1, ctas_per_sm=0, use_graph=0),
           dict(chunk_bytes=5000, stages=2, ctas_per_sm=1, use_graph=1),
           dict(chunk_bytes=70000, stages=3, ctas_per_sm=0, use_graph=1),
           dict(chunk_bytes=1 << 20, stages=4, ctas_per_sm=0, use_graph=0)]


@pytest.mark.parametrize("tuning", TUNINGS, ids=["default", "4k-s1", "5000-s2-graph",
                                                  "70k-s3-graph", "1m-s4"])
@pytest.mark.parametrize("shape", [(300, 0, 400), (40, 1000, 30000), (1000, 25, 80)],
                         ids=["mixed", "long", "reads"])
def test_ragged_insert_matches_per_record(sbf, cuda, oracle_mod, tuning, shape):
    n_records, lo, hi = shape
    rng = np.random.default_rng(n_records * 7 + hi)
    seq, ranges = _batch(rng, n_records, lo, hi)
    bits = 1 << 20
    f = sbf.Filter(bits, **K31)
    rep = f.ragged_insert(seq, ranges, tuning=tuning)
    o, w = _oracle_words(oracle_mod, bits, seq, ranges)
    np.testing.assert_array_equal(f.words_host(), w)
    _, recs = sbf.normalize_record_batch(31, seq, ranges)
    assert rep.records_indexed == n_records
    assert rep.indexed_bases == sum(n for _, n in ranges)
    assert rep.inserted_kmers == sum(r.valid_kmers for r in recs)


@pytest.mark.parametrize("tuning", TUNINGS[:3], ids=["default", "4k-s1", "5000-s2-graph"])
@pytest.mark.parametrize("shape", [(500, 0, 300), (30, 2000, 40000)], ids=["mixed", "long"])
def test_ragged_query_matches_per_record(sbf, cuda, oracle_mod, tuning, shape):
    n_records, lo, hi = shape
    rng = np.random.default_rng(n_records + lo + 11)
    seq, ranges = _batch(rng, n_records, lo, hi)
    bits = 1 << 18
    f = sbf.Filter(bits, **K31)
    f.ragged_insert(seq, ranges[::2])
    words = f.words_host()
    o = oracle_mod.Oracle(**K31)
    hits, rep = f.ragged_query(seq, ranges, tuning=tuning)
    assert hits.size == max(seq.size - 30, 0)
    covered = np.zeros(hits.size, bool)
    valid = positive = 0
    _, recs = sbf.normalize_record_batch(31, seq, ranges)
    for (off, n), rec in zip(ranges, recs):
        if n < 31:
            continue
        want = o.contains(words, seq[off:off + n])
        np.testing.assert_array_equal(hits[off:off + n - 30], want)
        covered[off:off + n - 30] = True
        positive += int(want.sum())
        valid += rec.valid_kmers
    assert not hits[~covered].any(), "windows outside every record must read 0"
    assert rep.queried_kmers == valid
    assert rep.positive_kmers == positive
    assert rep.records_queried == n_records


def test_ragged_device_entry_points(sbf, cuda, oracle_mod):
    torch = cuda
    rng = np.random.default_rng(5)
    seq, ranges = _batch(rng, 200, 0, 2000)
    bits = 1 << 20
    f = sbf.Filter(bits, **K31)
    d_seq = torch.from_numpy(seq.copy()).cuda()
    d_rng = torch.from_numpy(np.asarray(ranges, np.uint64).view(np.int64).reshape(-1, 2)).cuda()
    counts = torch.zeros(2, dtype=torch.int64, device="cuda")
    f.ragged_insert_async(d_seq, d_rng, counts)
    torch.cuda.synchronize()
    o, w = _oracle_words(oracle_mod, bits, seq, ranges)
    np.testing.assert_array_equal(f.words_host(), w)
    _, recs = sbf.normalize_record_batch(31, seq, ranges)
    assert int(counts[0]) == sum(r.valid_kmers for r in recs)
    out = torch.full((seq.size - 30,), 7, dtype=torch.uint8, device="cuda")
    counts.zero_()
    f.ragged_contains_async(d_seq, d_rng, out, counts)
    torch.cuda.synchronize()
    h = out.cpu().numpy()
    host_hits, rep = f.ragged_query(seq, ranges)
    np.testing.assert_array_equal(h, host_hits)
    assert int(counts[1]) == rep.positive_kmers == int(h.sum())
    with pytest.raises(sbf.SbfError):
        f.ragged_contains_async(d_seq, d_rng, out[:-1])


def test_ragged_equals_plain_per_record_launches(sbf, cuda):
    """The baseline the ragged form replaces: one insert_sequence per record."""
    rng = np.random.default_rng(9)
    seq, ranges = _batch(rng, 120, 10, 3000, gaps=False, alphabet=b"ACGT")
    a = sbf.Filter(1 << 22, **K31)
    b = sbf.Filter(1 << 22, **K31)
    a.ragged_insert(seq, ranges)
    for off, n in ranges:
        b.insert_sequence(seq[off:off + n])
    np.testing.assert_array_equal(a.words_host(), b.words_host())
    hits, _ = a.ragged_query(seq, ranges)
    for off, n in ranges:
        if n >= 31:
            np.testing.assert_array_equal(hits[off:off + n - 30], b.contains_sequence(seq[off:off + n]))


def test_ragged_edge_cases(sbf, cuda, oracle_mod):
    f = sbf.Filter(1 << 16, **K31)
    # no records, short buffers, records shorter than k
    rep = f.ragged_insert(np.zeros(0, np.uint8), [])
    assert rep.inserted_kmers == 0
    seq = np.frombuffer(b"ACGT" * 20, np.uint8)
    rep = f.ragged_insert(seq, [])
    assert rep.inserted_kmers == 0 and not f.words_host().any()
    rep = f.ragged_insert(seq, [(0, 30), (30, 30)])
    assert rep.inserted_kmers == 0 and not f.words_host().any()
    hits, qrep = f.ragged_query(seq, [(0, 30), (30, 30)])
    assert not hits.any() and qrep.queried_kmers == 0
    # one record exactly k long, ending at the buffer end
    rep = f.ragged_insert(seq, [(80 - 31, 31)])
    assert rep.inserted_kmers == 1
    with pytest.raises(sbf.SbfError):
        f.ragged_insert(seq, [(10, 5), (0, 5)])  # unsorted
    with pytest.raises(sbf.SbfError):
        f.ragged_insert(seq, [(70, 20)])  # out of bounds
    with pytest.raises(sbf.SbfError):
        f.ragged_insert(seq, [(0, 40)], tuning=dict(chunk_bytes=100, stages=2, ctas_per_sm=0,
                                                    use_graph=0))


def test_ragged_autotune_persists(sbf, cuda, oracle_mod, tmp_path, monkeypatch):
    table = tmp_path / "tune" / "ragged.tsv"
    monkeypatch.setenv("SBF_TUNE_TABLE", str(table))
    rng = np.random.default_rng(21)
    seq, ranges = _batch(rng, 400, 50, 3000, gaps=False)
    bits = 1 << 21
    f = sbf.Filter(bits, **K31)
    assert f.ragged_tuning_lookup(seq.size, len(ranges), query=False) is None
    t = f.ragged_autotune(seq, ranges, query=False, sample_bytes=1 << 18)
    assert table.exists() and t.stages in (2, 3)
    got = f.ragged_tuning_lookup(seq.size, len(ranges), query=False)
    assert got is not None and got.as_dict() == t.as_dict()
    f.ragged_insert(seq, ranges)  # tuned entry used
    o, w = _oracle_words(oracle_mod, bits, seq, ranges)
    np.testing.assert_array_equal(f.words_host(), w)
    tq = f.ragged_autotune(seq, ranges, query=True, sample_bytes=1 << 18)
    hits, _ = f.ragged_query(seq, ranges)
    hits2, _ = f.ragged_query(seq, ranges, tuning=tq)
    np.testing.assert_array_equal(hits, hits2)


@pytest.mark.parametrize("tuning", TUNINGS[:4], ids=["default", "4k-s1", "5000-s2-graph",
                                                     "70k-s3-graph"])
def test_ragged_query_bits_match_bytes(sbf, cuda, tuning):
    """The bit-packed ragged query equals the byte query bit for bit, across
    chunk boundaries (chunks hold a multiple of 32 windows)."""
    rng = np.random.default_rng(77)
    seq, ranges = _batch(rng, 400, 0, 3000)
    f = sbf.Filter(1 << 20, **K31)
    f.ragged_insert(seq, ranges[::3])
    hits, rep = f.ragged_query(seq, ranges, tuning=tuning)
    words, rep_b = f.ragged_query_bits(seq, ranges, tuning=tuning)
    b = np.packbits(hits.astype(np.uint8), bitorder="little")
    b = np.concatenate([b, np.zeros(words.size * 4 - b.size, np.uint8)])
    np.testing.assert_array_equal(words, b.view(np.uint32))
    assert rep_b.positive_kmers == rep.positive_kmers and rep_b.queried_kmers == rep.queried_kmers
    assert rep.positive_kmers > 0


def test_ragged_pinned_range_tables(sbf, cuda):
    """Pinned record tables are uploaded slice by slice without a host copy;
    results equal the pageable-table path."""
    torch = cuda
    rng = np.random.default_rng(81)
    seq, ranges = _batch(rng, 600, 0, 400)
    r = np.asarray(ranges, np.uint64)
    pinned = torch.empty(r.shape, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    pinned[:] = r
    small = dict(chunk_bytes=4096, stages=2, ctas_per_sm=0, use_graph=0)
    a = sbf.Filter(1 << 20, **K31)
    b = sbf.Filter(1 << 20, **K31)
    a.ragged_insert(seq, r[::2], tuning=small)
    b.ragged_insert(seq, np.ascontiguousarray(pinned[::2]), tuning=small)
    np.testing.assert_array_equal(a.words_host(), b.words_host())
    ha, ra = a.ragged_query(seq, r, tuning=small)
    hb, rb = a.ragged_query(seq, pinned, tuning=small)
    np.testing.assert_array_equal(ha, hb)
    assert ra.positive_kmers == rb.positive_kmers > 0
