"""Host expansion of bit-packed query results into one byte per window (CPU).

Host-output queries download one bit per window and expand it on host
threads; the bytes must equal the one-byte-per-window layout of
contains_sequence (include/cusbf/filter.cuh:514) for every length and output
alignment.
"""
import numpy as np
import pytest


def _expected(words, n):
    return np.unpackbits(words.view(np.uint8), bitorder="little")[:n]


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 1000, 4096 * 32 * 3 + 17])
@pytest.mark.parametrize("shift", [0, 1, 13, 31])
@pytest.mark.parametrize("threads", [1, 3, 8])
def test_expand_matches_unpackbits(sbf, n, shift, threads):
    rng = np.random.default_rng(n * 131 + shift * 7 + threads)
    words = rng.integers(0, 2**32, size=max((n + 31) // 32, 1), dtype=np.uint32)
    buf = np.full(n + 64 + 64, 0xEE, np.uint8)
    # Start the output `shift` bytes past a 64-byte boundary.
    base = (-buf.ctypes.data) % 64
    out = buf[base + shift: base + shift + n]
    if n == 0:
        assert sbf.expand_result_bits(words, 0, out=buf[:1], threads=threads).size == 0
        return
    got = sbf.expand_result_bits(words, n, out=out, threads=threads)
    assert np.array_equal(got, _expected(words, n))
    # Bytes around the output are untouched.
    assert (buf[:base + shift] == 0xEE).all()
    assert (buf[base + shift + n:] == 0xEE).all()


def test_expand_rejects_short_spans(sbf):
    with pytest.raises(ValueError):
        sbf.expand_result_bits(np.zeros(1, np.uint32), 33)
    with pytest.raises(ValueError):
        sbf.expand_result_bits(np.zeros(2, np.uint32), 40, out=np.zeros(39, np.uint8))
