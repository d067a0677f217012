"""The engine against the committed golden fixtures (tests/golden/): filter
words and query bytes generated by the reference's own arithmetic
(oracle/_ref, tests/golden/make_golden.py) for six DNA configurations and the
protein and DNA-triplet alphabets.  Needs no oracle at run time."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["k31_uniform", "k31_invalid", "k31_h8", "k31_h16", "k21", "k5", "prot5", "trip3"]


@pytest.mark.parametrize("name", NAMES)
def test_engine_equals_golden(sbf, cuda, name):
    z = np.load(os.path.join(GOLDEN, "k31_small.npz"))
    k, s, m, h, bits = (int(x) for x in z[f"{name}__cfg"])
    alphabet = int(z[f"{name}__alphabet"][0])
    f = sbf.Filter(bits, k=k, s=s, m=m, hashes=h, alphabet=alphabet)
    f.insert_sequence(z[f"{name}__insert"])
    np.testing.assert_array_equal(f.words_host(), z[f"{name}__words"])
    np.testing.assert_array_equal(f.contains_sequence(z[f"{name}__query"]), z[f"{name}__hits"])
    f.close()
