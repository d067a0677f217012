"""Per-record counts computed in the ragged query kernel's epilogue
(sbf_ragged_contains_counts_async) equal the reference's second pass
(count_positive_kmers_per_record, detail/count_positive_kmers.cuh:21-45): the
sum of the record's hit bytes, and its valid windows.  Checked against the
oracle record by record, with and without hit bytes, at odd output
alignments, and for the layouts that stress the record walk: empty records
sharing an offset, records shorter than k, many records per 32-window strip,
N runs that empty whole strips, and records spanning many tiles."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)
VALID = np.zeros(256, bool)
VALID[np.frombuffer(b"ACGTacgt", np.uint8)] = True


def _valid_windows(seq, k=31):
    if seq.size < k:
        return 0
    bad = np.concatenate([[0], np.cumsum(~VALID[seq])])
    return int(((bad[k:] - bad[:-k]) == 0).sum())


def _layout(rng, kind):
    parts, ranges, pos = [], [], 0

    def put(n, alphabet=b"ACGT", gap=0):
        nonlocal pos
        if gap:
            parts.append(random_dna(rng, gap, b"ACGT"))
            pos += gap
        parts.append(random_dna(rng, n, alphabet))
        ranges.append((pos, n))
        pos += n

    if kind == "mixed":
        for _ in range(400):
            put(int(rng.integers(0, 600)), b"ACGTACGTACGTACGTN",
                gap=int(rng.integers(1, 20)) if rng.random() < 0.3 else 0)
    elif kind == "tiny":  # several records per strip
        for _ in range(3000):
            put(int(rng.integers(28, 45)))
    elif kind == "empty-shared":  # empty records at the offset of the next one
        for i in range(300):
            if i % 3 == 0:
                ranges.append((pos, 0))
            put(int(rng.integers(0, 300)))
    elif kind == "n-runs":  # N runs longer than a strip inside records
        for _ in range(40):
            a = random_dna(rng, int(rng.integers(100, 3000)))
            a[int(rng.integers(0, 50)):][:int(rng.integers(40, 400))] = ord("N")
            parts.append(a)
            ranges.append((pos, a.size))
            pos += a.size
    elif kind == "long":  # records spanning many 8192-window tiles
        for _ in range(6):
            put(int(rng.integers(20_000, 90_000)), gap=int(rng.integers(0, 40)))
    else:
        raise ValueError(kind)
    parts.append(random_dna(rng, 7, b"ACGT"))
    return np.concatenate(parts), ranges


@pytest.mark.parametrize("kind", ["mixed", "tiny", "empty-shared", "n-runs", "long"])
@pytest.mark.parametrize("align", [None, 0, 3])
def test_counts_match_oracle(sbf, cuda, oracle_mod, kind, align):
    torch = cuda
    kinds = ["mixed", "tiny", "empty-shared", "n-runs", "long"]
    rng = np.random.default_rng(10 * kinds.index(kind) + (5 if align is None else align))
    seq, ranges = _layout(rng, kind)
    bits = 1 << 18
    f = sbf.Filter(bits, **K31)
    f.ragged_insert(seq, [r for i, r in enumerate(ranges) if i % 2 == 0])
    words = f.words_host()
    o = oracle_mod.Oracle(**K31)
    n = len(ranges)
    want_valid = np.zeros(n, np.uint64)
    want_pos = np.zeros(n, np.uint64)
    for i, (off, ln) in enumerate(ranges):
        r = seq[off:off + ln]
        want_valid[i] = _valid_windows(r)
        if ln >= 31:
            want_pos[i] = int(o.contains(words, r).sum())
    d_seq = torch.from_numpy(seq.copy()).cuda()
    d_rng = torch.from_numpy(np.asarray(ranges, np.uint64).view(np.int64).reshape(-1, 2)).cuda()
    rv = torch.full((n,), 99, dtype=torch.int64, device="cuda")
    rp = torch.full((n,), 99, dtype=torch.int64, device="cuda")
    counts = torch.zeros(2, dtype=torch.int64, device="cuda")
    w = seq.size - 30
    out = None
    if align is not None:
        buf = torch.full((w + 16,), 7, dtype=torch.uint8, device="cuda")
        out = buf[align:align + w]
    f.ragged_contains_counts_async(d_seq, d_rng, rv, rp, d_out=out, d_counts=counts)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(rv.cpu().numpy().astype(np.uint64), want_valid)
    np.testing.assert_array_equal(rp.cpu().numpy().astype(np.uint64), want_pos)
    assert int(counts[0]) == int(want_valid.sum())
    assert int(counts[1]) == int(want_pos.sum())
    if out is not None:
        ref = torch.zeros(w, dtype=torch.uint8, device="cuda")
        f.ragged_contains_async(d_seq, d_rng, ref)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())


def test_counts_edge_cases(sbf, cuda):
    torch = cuda
    f = sbf.Filter(1 << 16, **K31)
    seq = np.frombuffer(b"ACGT" * 40, np.uint8)
    d_seq = torch.from_numpy(seq.copy()).cuda()
    f.insert_sequence(seq)
    # no records: nothing to count
    empty = torch.zeros((0, 2), dtype=torch.int64, device="cuda")
    z = torch.zeros(0, dtype=torch.int64, device="cuda")
    f.ragged_contains_counts_async(d_seq, empty, z, z)
    # records shorter than k, and one exactly k long at the end
    rng_ = [(0, 30), (30, 0), (30, 30), (160 - 31, 31)]
    d_rng = torch.tensor(rng_, dtype=torch.int64, device="cuda")
    rv = torch.full((4,), 5, dtype=torch.int64, device="cuda")
    rp = torch.full((4,), 5, dtype=torch.int64, device="cuda")
    f.ragged_contains_counts_async(d_seq, d_rng, rv, rp)
    torch.cuda.synchronize()
    assert rv.tolist() == [0, 0, 0, 1] and rp.tolist() == [0, 0, 0, 1]
    # too-small output span, and count arrays shorter than the record table
    with pytest.raises(sbf.SbfError):
        f.ragged_contains_counts_async(d_seq, d_rng, rv, rp,
                                       d_out=torch.zeros(10, dtype=torch.uint8, device="cuda"))
    with pytest.raises(ValueError):
        f.ragged_contains_counts_async(d_seq, d_rng, rv[:3], rp)
