"""Record-batch host logic (CPU): normalisation and query layout.

Known answers restate the reference's host tests
(tests/test_query_layout.cpp, tests/test_normalized_record_batch.cpp of
tdortman/cuSBF, both with Config<3, 2, 2, 4>).
"""
import numpy as np
import pytest

from conftest import random_dna


def test_layout_hit_spans(sbf):
    # test_query_layout.cpp:9-53
    recs = [sbf.NormalizedRecord(0, 0, 6, 1), sbf.NormalizedRecord(1, 6, 8, 2)]
    layout, total = sbf.query_layout(3, recs)
    assert total == 13
    assert (layout[0].hit_offset, layout[0].hit_count, layout[0].valid_kmers) == (0, 4, 1)
    assert (layout[1].hit_offset, layout[1].hit_count, layout[1].valid_kmers) == (7, 6, 2)
    assert (layout[1].record_index, layout[1].input_offset, layout[1].size) == (1, 6, 8)


def test_layout_valid_separate_from_hits(sbf):
    # test_query_layout.cpp:56-69
    layout, total = sbf.query_layout(3, [sbf.NormalizedRecord(0, 0, 14, 3)])
    assert total == 12 and layout[0].valid_kmers == 3 and layout[0].hit_count == 12


def test_layout_boundary_windows(sbf):
    # test_query_layout.cpp:71-84
    layout, total = sbf.query_layout(3, [sbf.NormalizedRecord(0, 0, 4, 0),
                                         sbf.NormalizedRecord(1, 4, 4, 0)])
    assert (layout[0].hit_count, layout[1].hit_count, total) == (2, 2, 7)


def test_normalize_injects_separators(sbf):
    # test_normalized_record_batch.cpp:10-18, :29-39
    seq, recs = sbf.normalize_record_batch(3, "ACGTACGTACGT", [(0, 4), (4, 4)])
    assert len(recs) == 2 and seq.size > 8
    assert sum(r.valid_kmers for r in recs) == 4
    assert seq.tobytes() == b"ACGTNACGT"
    assert (recs[0].record_index, recs[1].record_index) == (0, 1)
    assert (recs[0].input_offset, recs[1].input_offset) == (0, 4)


def test_normalize_rejects_overlap(sbf):
    # test_normalized_record_batch.cpp:20-27
    with pytest.raises(sbf.SbfError) as e:
        sbf.normalize_record_batch(3, "ACGTACGT", [(4, 4), (0, 4)])
    assert e.value.category == "invalid_argument"
    with pytest.raises(sbf.SbfError):
        sbf.validate_record_batch(8, [(0, 4), (4, 5)])


def test_validate_large_batch_reports_first_bad_record(sbf):
    # Batches of millions of records are checked in segments on several host
    # threads; the result and message must be those of a serial scan.
    n, size = 6_000_000, 10
    r = np.empty((n, 2), np.uint64)
    r[:, 0] = np.arange(n, dtype=np.uint64) * size
    r[:, 1] = size
    total = n * size
    sbf.validate_record_batch(total, r)
    # Overlap across a segment boundary (segments start at multiples of n/3).
    bad = r.copy()
    bad[1_999_999, 1] = size + 1
    with pytest.raises(sbf.SbfError, match="ordered and non-overlapping"):
        sbf.validate_record_batch(total, bad)
    # Two faults: the earlier one (out of bounds) decides the message.
    bad = r.copy()
    bad[4_000_000, 1] = total
    bad[5_500_000, 0] -= 1
    with pytest.raises(sbf.SbfError, match="exceeds the source sequence"):
        sbf.validate_record_batch(total, bad)
    bad = r.copy()
    bad[5_999_999, 0] -= 1
    with pytest.raises(sbf.SbfError, match="ordered and non-overlapping"):
        sbf.validate_record_batch(total, bad)


def _py_normalize(seq, ranges, k):
    out, recs = bytearray(), []
    for i, (o, n) in enumerate(ranges):
        if len(out):
            out += b"N"
        rec = bytes(seq[o:o + n])
        out += rec
        ok = [(c & 0xDF) in b"ACGT" for c in rec]
        valid = sum(all(ok[p:p + k]) for p in range(0, max(0, n - k + 1)))
        recs.append((i, o, n, valid))
    return bytes(out), recs


def test_normalize_matches_restatement(sbf):
    rng = np.random.default_rng(3)
    seq = random_dna(rng, 5000, b"ACGTACGTACGTNn")
    for _ in range(20):
        cuts = np.sort(rng.choice(5000, size=int(rng.integers(1, 30)) * 2, replace=False))
        ranges = [(int(cuts[i]), int(cuts[i + 1] - cuts[i])) for i in range(0, len(cuts), 2)]
        if rng.random() < 0.5:
            ranges.insert(0, (0, 0))  # empty leading record: no separator before the next
        ranges.sort()
        for k in (3, 5, 31):
            joined, recs = sbf.normalize_record_batch(k, seq, ranges)
            want_seq, want_recs = _py_normalize(seq, ranges, k)
            assert joined.tobytes() == want_seq
            assert [(r.record_index, r.input_offset, r.size, r.valid_kmers) for r in recs] == want_recs
            # estimate_normalized_batch_bytes (normalized_record_batch.hpp:179-194)
            # counts a separator before every record but the first even when
            # earlier records are empty: an upper bound of the joined length.
            est = 0
            for i, (_, n) in enumerate(ranges):
                if i != 0 or est != 0:
                    est += 1
                est += n
            assert sbf.normalized_batch_bytes(ranges) == est >= len(want_seq)
