"""Host-output queries that download one bit per window and expand it on
host threads return the same bytes as downloading the bytes, and as the
device-output path, for multi-chunk inputs, misaligned and pageable outputs,
dense input and ragged batches."""
import ctypes as C

import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def _filter(sbf, monkeypatch, expand, rng):
    # The choice is made once per filter, at its first host-output query.
    monkeypatch.setenv("SBF_HOST_EXPAND", expand)
    f = sbf.Filter(1 << 22, **K31)
    ref = random_dna(rng, 2_000_000, b"ACGTACGTACGTN")
    f.insert_sequence(ref)
    return f, ref


def _query_into(sbf, f, q, out):
    """sbf_contains_sequence into a caller-supplied (possibly misaligned) span."""
    qa = np.ascontiguousarray(q)
    rc = sbf._lib.sbf_contains_sequence(f._h, qa.ctypes.data, qa.size, out.ctypes.data, out.size,
                                        None)
    assert rc == 0, sbf._lib.sbf_last_error_message()


@pytest.mark.parametrize("chunk", ["65536", "1048576", None])
def test_plain_expand_equals_bytes(sbf, cuda, monkeypatch, chunk):
    torch = cuda
    if chunk:
        monkeypatch.setenv("SBF_HOST_CHUNK_BYTES", chunk)
    rng = np.random.default_rng(11)
    results = {}
    for expand in ("0", "1"):
        f, ref = _filter(sbf, monkeypatch, expand, np.random.default_rng(11))
        q = np.concatenate([ref[:1_500_000], random_dna(rng, 2_400_013, b"ACGTACGTN")])
        n = f.kmer_count(q.size)
        buf = np.full(n + 64, 0xEE, np.uint8)
        for shift in (0, 5):
            out = buf[shift:shift + n]
            _query_into(sbf, f, q, out)
            assert (buf[shift + n:] == 0xEE).all()
            results[(expand, shift)] = out.copy()
            buf[:] = 0xEE
        d_q = torch.from_numpy(q).cuda()
        d_out = torch.empty(n, dtype=torch.uint8, device="cuda")
        f.contains_sequence_async(d_q, d_out)
        torch.cuda.synchronize()
        results[(expand, "dev")] = d_out.cpu().numpy()
        rng = np.random.default_rng(11)
    want = results[("0", "dev")]
    assert want.any() and not want.all()
    for key, got in results.items():
        np.testing.assert_array_equal(got, want, err_msg=str(key))


def test_dense_expand_equals_bytes(sbf, cuda, monkeypatch):
    monkeypatch.setenv("SBF_HOST_CHUNK_BYTES", "65536")
    rng = np.random.default_rng(4)
    out = {}
    for expand in ("0", "1"):
        f, ref = _filter(sbf, monkeypatch, expand, np.random.default_rng(4))
        q = np.concatenate([ref[:900_000], random_dna(rng, 700_003)])
        packed = sbf.pack_dense_sequence(q)
        out[expand] = f.contains_dense_packed(packed, q.size)
        rng = np.random.default_rng(4)
    np.testing.assert_array_equal(out["1"], out["0"])


@pytest.mark.parametrize("chunk", [1 << 20, 0])
def test_ragged_expand_equals_bytes(sbf, cuda, monkeypatch, chunk):
    torch = cuda
    rng = np.random.default_rng(8)
    lens = rng.integers(20, 400, size=30_000)
    gaps = rng.integers(0, 3, size=lens.size)
    off = np.cumsum(np.concatenate([[0], lens[:-1] + gaps[:-1]]))
    total = int(off[-1] + lens[-1] + 7)
    ranges = np.stack([off, lens], axis=1).astype(np.uint64)
    res = {}
    for expand in ("0", "1"):
        f, ref = _filter(sbf, monkeypatch, expand, np.random.default_rng(8))
        head = ref[:min(total // 2, ref.size)]
        tail = random_dna(np.random.default_rng(99), total - head.size)
        seq = np.concatenate([head, tail])
        assert seq.size == total
        tuning = sbf.RaggedTuning(chunk, 3, 0, 0) if chunk else None
        n = f.kmer_count(seq.size)
        buf = np.full(n + 40, 0xEE, np.uint8)
        hits, rep = f.ragged_query(seq, ranges, out=buf[3:3 + n], tuning=tuning)
        assert (buf[:3] == 0xEE).all() and (buf[3 + n:] == 0xEE).all()
        res[expand] = (hits.copy(), rep.positive_kmers, rep.queried_kmers)
        d_seq = torch.from_numpy(seq).cuda()
        d_rng = torch.from_numpy(ranges.view(np.int64)).cuda()
        d_out = torch.empty(n, dtype=torch.uint8, device="cuda")
        f.ragged_contains_async(d_seq, d_rng, d_out)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(hits, d_out.cpu().numpy())
    np.testing.assert_array_equal(res["1"][0], res["0"][0])
    assert res["1"][1:] == res["0"][1:]
    assert res["0"][1] > 0
