"""The oracle itself, pinned (CPU only).

1. Against the reference's own known-answer tests (tests/test_bloom_filter.cu
   of tdortman/cuSBF, configurations of tests/test_support.cuh:20-22).
2. Against the golden fixtures of tests/golden/, produced by the reference's
   own arithmetic (oracle/_ref, see tests/golden/make_golden.py).
3. Against oracle/_ref directly on fresh random inputs, when it is present.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import random_dna

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _o(oracle_mod, k, s, m, h=4, alphabet=0):
    return oracle_mod.Oracle(k, s, m, h, alphabet)


def test_dna_invalid_windows(oracle_mod):
    # test_bloom_filter.cu:91-101
    o = _o(oracle_mod, 5, 4, 3)
    w = o.new_words(1 << 12)
    seq = "ACGTNACGTACGTA"
    assert o.insert(w, seq) == 10
    assert list(o.contains(w, seq)) == [0, 0, 0, 0, 0, 1, 1, 1, 1, 1]


def test_no_false_negatives_and_idempotence(oracle_mod):
    # test_bloom_filter.cu:10-20, :103-115
    o = _o(oracle_mod, 5, 4, 3)
    w = o.new_words(1 << 12)
    seq = "ACGTACGTACGTACGT"
    assert o.insert(w, seq) == 12
    assert o.contains(w, seq).all()
    before = w.copy()
    o.insert(w, seq)
    np.testing.assert_array_equal(before, w)


def test_short_and_lowercase(oracle_mod):
    # test_bloom_filter.cu:117-128, :228-241
    o = _o(oracle_mod, 5, 4, 3)
    w = o.new_words(1 << 12)
    assert o.insert(w, "ACGT") == 0
    assert o.contains(w, "ACGT").size == 0
    o.insert(w, "acgtacgtacgtacgt")
    assert o.contains(w, "ACGTACGTACGTACGT").all()


def test_protein_and_triplet(oracle_mod):
    # test_bloom_filter.cu:267-277 (protein), :317-327, :329-339 (triplet)
    p = _o(oracle_mod, 5, 4, 3, alphabet=oracle_mod.ALPHABET_PROTEIN)
    w = p.new_words(1 << 12)
    seq = "ACDE*ACDEFGHI"
    p.insert(w, seq)
    assert list(p.contains(w, seq)) == [0, 0, 0, 0, 0, 1, 1, 1, 1]
    t = _o(oracle_mod, 3, 2, 2, alphabet=oracle_mod.ALPHABET_DNA_TRIPLET)
    w = t.new_words(1 << 12)
    seq = "ACGTACNNNGGGTTTAAA"
    t.insert(w, seq)
    assert list(t.contains(w, seq)) == [0, 0, 0, 1]
    w = t.new_words(1 << 12)
    seq = "ACGTACGTTAAACCCGGGTTTAA"
    assert t.insert(w, seq) == 5
    assert t.contains(w, seq).all()


def test_separator_windows(oracle_mod):
    # test_bloom_filter.cu:373-422: 8 ones, 5 zeros, 8 ones.
    o = _o(oracle_mod, 5, 4, 3)
    w = o.new_words(1 << 14)
    r1, r2 = "ACGTACGTACGT", "TTGGAACCTTGG"
    o.insert(w, r1)
    o.insert(w, r2)
    assert list(o.contains(w, r1 + "N" + r2)) == [1] * 8 + [0] * 5 + [1] * 8


def test_dense_matches_bytes(oracle_mod):
    # test_bloom_filter.cu:22-38
    o = _o(oracle_mod, 5, 4, 3)
    seq = "ACGTACGTACGTACGTACGTACGT"
    packed = o.pack_dense(seq)
    w = o.new_words(1 << 12)
    o.insert_dense(w, packed, len(seq))
    hits = o.contains_dense(w, packed, len(seq))
    assert hits.all() and hits.size == len(seq) - 4
    np.testing.assert_array_equal(hits, o.contains(w, seq))


def test_shard_count(oracle_mod):
    # filter.cuh:108-118
    ns = oracle_mod.num_shards
    assert ns(0) == 1 and ns(1) == 1 and ns(256) == 1 and ns(257) == 2
    assert ns(1 << 28) == 1 << 20
    assert ns(int(85.7 * 1_999_970)) == 1 << 20


@pytest.mark.parametrize("name", ["k31_uniform", "k31_invalid", "k31_h8", "k31_h16", "k21", "k5",
                                  "prot5", "trip3"])
def test_golden_vectors(oracle_mod, name):
    """Fixtures from the reference's own arithmetic (oracle/_ref), including
    the protein and DNA-triplet alphabets."""
    z = np.load(os.path.join(GOLDEN, "k31_small.npz"))
    k, s, m, h, bits = (int(x) for x in z[f"{name}__cfg"])
    alphabet = int(z[f"{name}__alphabet"][0])
    o = _o(oracle_mod, k, s, m, h, alphabet)
    w = o.new_words(bits)
    o.insert(w, z[f"{name}__insert"])
    np.testing.assert_array_equal(w, z[f"{name}__words"])
    np.testing.assert_array_equal(o.contains(w, z[f"{name}__query"]), z[f"{name}__hits"])


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_golden_digest_plain_small(oracle_mod):
    """The plain-method small workload (2 Mbp, 85.7 bits/k-mer) digests."""
    from workloads.synthetic import uniform_dna

    d = json.load(open(os.path.join(GOLDEN, "digests.json")))["plain_small"]
    ins = uniform_dna(2_000_000, seed=42)
    fresh = uniform_dna(2_000_000, seed=1337)
    o = oracle_mod.Oracle()
    w = o.new_words(d["requested_bits"])
    o.insert(w, ins)
    assert _sha(w) == d["words_sha256"]
    assert _sha(o.contains(w, ins)) == d["hits_positive_sha256"]
    assert _sha(o.contains(w, fresh)) == d["hits_fresh_sha256"]


def test_refcpu_cross_check(oracle_mod):
    if not oracle_mod.RefCpu.available():
        pytest.skip("oracle/_ref is built only where the reference sources are present")
    rng = np.random.default_rng(2024)
    for key in oracle_mod.REF_CONFIGS:
        k, s, m, h, alpha = key
        letters = {0: b"ACGTacgtN", 1: b"ACGTN", 2: b"ACDEFGHIKLMNPQRSTVWY*"}[alpha]
        seq = random_dna(rng, 5000, letters)
        o = oracle_mod.Oracle(k, s, m, h, alpha)
        r = oracle_mod.RefCpu(k, s, m, h, alpha)
        for bits in (1 << 10, 1 << 18):
            w1, w2 = o.new_words(bits), o.new_words(bits)
            o.insert(w1, seq)
            r.insert(w2, seq)
            np.testing.assert_array_equal(w1, w2)
            q = np.concatenate([seq[:2000], random_dna(rng, 3000, letters)])
            np.testing.assert_array_equal(o.contains(w1, q), r.contains(w2, q))


def test_threads_do_not_change_results(oracle_mod):
    rng = np.random.default_rng(8)
    seq = random_dna(rng, 200_000, b"ACGTN")
    o = oracle_mod.Oracle()
    w1, w8 = o.new_words(1 << 20), o.new_words(1 << 20)
    o.insert(w1, seq, threads=1)
    o.insert(w8, seq, threads=8)
    np.testing.assert_array_equal(w1, w8)
    np.testing.assert_array_equal(o.contains(w1, seq, threads=1), o.contains(w8, seq, threads=8))
