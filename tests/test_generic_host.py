"""Host-side parts of the generic configurations (no GPU): dense packing for
every alphabet against the oracle, and the reference's Config rules
(config.cuh:76-118) enforced by sbf_filter_create before any device work."""
import numpy as np
import pytest

from conftest import random_dna

DNA, TRIPLET, PROTEIN = 0, 1, 2


@pytest.mark.parametrize("alphabet,width,bits", [(DNA, 1, 2), (PROTEIN, 1, 5), (TRIPLET, 3, 6)])
def test_dense_packing_matches_oracle(sbf, oracle_mod, alphabet, width, bits):
    rng = np.random.default_rng(alphabet)
    for n in (0, 1, 11, 12, 13, 31, 32, 33, 1000, 4097):
        if alphabet == PROTEIN:
            a = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWYxbz*- ", np.uint8)
            seq = a[rng.integers(0, a.size, n)]
        else:
            seq = random_dna(rng, n * width + (n % 3), b"ACGTacgtN")
        got = sbf.pack_dense_sequence(seq, alphabet=alphabet)
        o = oracle_mod.Oracle(k=1, s=1, m=1, hashes=4, alphabet=alphabet)
        want = o.pack_dense(seq)
        np.testing.assert_array_equal(got, want)
        per = 64 // bits
        assert sbf.Filter.dense_packed_word_count(seq.size // width, alphabet) == \
            (seq.size // width + per - 1) // per


@pytest.mark.parametrize("cfg", [
    dict(k=0, s=1, m=1, hashes=4, alphabet=DNA),
    dict(k=33, s=20, m=16, hashes=4, alphabet=DNA),
    dict(k=13, s=10, m=6, hashes=4, alphabet=PROTEIN),
    dict(k=11, s=8, m=5, hashes=4, alphabet=TRIPLET),
    dict(k=21, s=19, m=22, hashes=4, alphabet=DNA),
    dict(k=21, s=0, m=11, hashes=4, alphabet=DNA),
    dict(k=21, s=19, m=11, hashes=6, alphabet=DNA),
    dict(k=21, s=19, m=11, hashes=20, alphabet=DNA),
    dict(k=21, s=19, m=11, hashes=4, alphabet=7),
])
def test_invalid_configs_rejected(sbf, cfg):
    with pytest.raises(sbf.SbfError) as ei:
        sbf.Filter(1 << 16, **cfg)
    assert ei.value.status == sbf.ERR_INVALID_ARGUMENT


def test_normalize_protein_and_triplets(sbf):
    # write_record_boundary (normalized_record_batch.hpp:209-232): one
    # separator symbol between records -- '*' for proteins, "NNN" for triplets.
    seq, recs = sbf.normalize_record_batch(3, "ACDEFGHI", [(0, 4), (4, 4)], alphabet=PROTEIN)
    assert seq.tobytes() == b"ACDE*FGHI"
    assert [r.valid_kmers for r in recs] == [2, 2]
    seq, recs = sbf.normalize_record_batch(2, "ACGTACGGGTTT", [(0, 6), (6, 6)],
                                           alphabet=TRIPLET)
    assert seq.tobytes() == b"ACGTACNNNGGGTTT"
    assert [r.valid_kmers for r in recs] == [1, 1]
    assert sbf.normalized_batch_bytes([(0, 6), (6, 6)], alphabet=TRIPLET) == 15
    layout, total = sbf.query_layout(2, recs, alphabet=TRIPLET)
    assert (layout[0].hit_offset, layout[1].hit_offset) == (0, 3)
    assert (layout[0].hit_count, layout[1].hit_count, total) == (1, 1, 4)
    # an invalid triplet in a record (any of its three bytes) resets windows
    _, recs = sbf.normalize_record_batch(2, "ACGACGNGG", [(0, 9)], alphabet=TRIPLET)
    assert recs[0].valid_kmers == 1
    _, recs = sbf.normalize_record_batch(2, "ACGNACGGG", [(0, 9)], alphabet=TRIPLET)
    assert recs[0].valid_kmers == 0


def test_triplet_ranges_must_align(sbf):
    # filter.cuh:865-873
    with pytest.raises(sbf.SbfError):
        sbf.validate_record_batch(12, [(0, 4), (6, 6)], alphabet=TRIPLET)
    with pytest.raises(sbf.SbfError):
        sbf.normalize_record_batch(2, "ACGTACGTACGT", [(1, 6)], alphabet=TRIPLET)
    sbf.validate_record_batch(12, [(0, 6), (6, 6)], alphabet=TRIPLET)
