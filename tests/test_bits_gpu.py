"""Bit-packed query results equal the byte results bit for bit: bit i % 32 of
word i // 32 is window i's hit, and the bits after the last window are 0."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def _pack(hits: np.ndarray) -> np.ndarray:
    n_words = (hits.size + 31) // 32
    b = np.packbits(hits.astype(np.uint8), bitorder="little")
    b = np.concatenate([b, np.zeros(n_words * 4 - b.size, np.uint8)])
    return b.view(np.uint32)


def _filter(sbf, rng, bits=1 << 22):
    f = sbf.Filter(bits, **K31)
    ref = random_dna(rng, 3_000_000, b"ACGTACGTACGTN")
    f.insert_sequence(ref)
    return f, ref


@pytest.mark.parametrize("length", [31, 32, 62, 63, 64, 100, 8192 + 30, 8193 + 30, 100_003,
                                    1_000_000])
def test_device_bits_match_bytes(sbf, cuda, length):
    torch = cuda
    rng = np.random.default_rng(length)
    f, ref = _filter(sbf, rng)
    q = np.concatenate([ref[:length // 2], random_dna(rng, length - length // 2)])
    want = _pack(f.contains_sequence(q))
    for off in (0, 3):
        buf = torch.zeros(q.size + off, dtype=torch.uint8, device="cuda")
        buf[off:] = torch.from_numpy(q)
        n_words = want.size
        d_bits = torch.full((n_words + 2,), -1, dtype=torch.int32, device="cuda")
        f.contains_sequence_bits_async(buf[off:], d_bits[:n_words])
        torch.cuda.synchronize()
        got = d_bits.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got[:n_words], want)
        assert (got[n_words:] == 0xFFFFFFFF).all(), "words past the span must be untouched"


@pytest.mark.parametrize("chunk", ["4096", "65536", None])
def test_host_bits_pipeline(sbf, cuda, monkeypatch, chunk):
    if chunk:
        monkeypatch.setenv("SBF_HOST_CHUNK_BYTES", chunk)
    rng = np.random.default_rng(5)
    f, ref = _filter(sbf, rng)
    q = np.concatenate([ref[:400_000], random_dna(rng, 300_007)])
    np.testing.assert_array_equal(f.contains_sequence_bits(q), _pack(f.contains_sequence(q)))


def test_bits_errors(sbf, cuda):
    torch = cuda
    f = sbf.Filter(1 << 16, **K31)
    q = torch.from_numpy(random_dna(np.random.default_rng(1), 1000)).cuda()
    small = torch.zeros(30, dtype=torch.int32, device="cuda")  # needs 31 words
    with pytest.raises(sbf.SbfError):
        f.contains_sequence_bits_async(q, small)
    raw = torch.zeros(200, dtype=torch.uint8, device="cuda")
    with pytest.raises(sbf.SbfError):
        f.contains_sequence_bits_async(q, (raw.data_ptr() + 1, 196))  # misaligned


@pytest.mark.parametrize("cfg", [K31, dict(k=12, s=10, m=6, hashes=8, alphabet=2)],
                         ids=["k31", "protein12"])
@pytest.mark.parametrize("chunk", [None, "4096"])
def test_dense_bits_match_dense_bytes(sbf, cuda, monkeypatch, cfg, chunk):
    """Dense-packed input with bit-packed results (host pipeline and device
    entry point) equals the dense byte results."""
    torch = cuda
    if chunk:
        monkeypatch.setenv("SBF_HOST_CHUNK_BYTES", chunk)
    rng = np.random.default_rng(len(cfg) + (chunk is None))
    alphabet = cfg.get("alphabet", 0)
    if alphabet == 2:
        a = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)
        seq = a[rng.integers(0, a.size, 700_001)]
    else:
        seq = random_dna(rng, 700_001)
    f = sbf.Filter(1 << 22, **cfg)
    packed = sbf.pack_dense_sequence(seq, alphabet=alphabet)
    f.insert_dense_packed(packed[: packed.size // 3], (packed.size // 3) * (64 // (5 if alphabet else 2)))
    want = f.contains_dense_packed(packed, seq.size)
    assert want.any() and not want.all()
    got = f.contains_dense_packed_bits(packed, seq.size)
    np.testing.assert_array_equal(got, _pack(want))
    d_words = torch.from_numpy(packed.view(np.int64).copy()).cuda()
    d_bits = torch.full((got.size + 3,), -1, dtype=torch.int32, device="cuda")
    f.contains_dense_packed_bits_async(d_words, seq.size, d_bits[:got.size])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_bits[:got.size].cpu().numpy().view(np.uint32), got)
