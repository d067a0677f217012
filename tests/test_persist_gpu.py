"""Filter persistence on the GPU: save -> load gives the same words and the
same answers; mismatched or malformed files leave the filter unchanged."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def test_round_trip(sbf, cuda, tmp_path):
    rng = np.random.default_rng(1)
    seq = random_dna(rng, 2_000_000)
    f = sbf.Filter(1 << 24, **K31)
    f.insert_sequence(seq)
    path = tmp_path / "f.sbf"
    f.save(path)
    assert path.stat().st_size == 40 + f.num_shards() * 32
    g = sbf.Filter.load(path)
    np.testing.assert_array_equal(g.words_host(), f.words_host())
    q = random_dna(rng, 100_000)
    np.testing.assert_array_equal(g.contains_sequence(seq[:50_000]), f.contains_sequence(seq[:50_000]))
    np.testing.assert_array_equal(g.contains_sequence(q), f.contains_sequence(q))


def test_rejects_mismatch_and_truncation(sbf, cuda, tmp_path):
    rng = np.random.default_rng(2)
    f = sbf.Filter(1 << 20, **K31)
    f.insert_sequence(random_dna(rng, 100_000))
    path = tmp_path / "f.sbf"
    f.save(path)
    other = sbf.Filter(1 << 21, **K31)
    other.insert_sequence(random_dna(rng, 1000))
    before = other.words_host()
    with pytest.raises(sbf.SbfError):
        other.load_words(path)  # another size
    np.testing.assert_array_equal(other.words_host(), before)
    k21 = sbf.Filter(1 << 20, k=21, s=19, m=11, hashes=4)
    with pytest.raises(sbf.SbfError):
        k21.load_words(path)  # another configuration
    data = path.read_bytes()
    short = tmp_path / "short.sbf"
    short.write_bytes(data[:-32])
    same = sbf.Filter(1 << 20, **K31)
    same.insert_sequence(random_dna(rng, 1000))
    before = same.words_host()
    with pytest.raises(sbf.SbfError):
        same.load_words(short)
    np.testing.assert_array_equal(same.words_host(), before)
