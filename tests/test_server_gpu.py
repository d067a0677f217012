"""Request server (sbf_server_*): continuous batching of mixed insert and
query requests gives, for every request, exactly the result of executing the
requests one at a time in arrival order."""
import threading

import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def _mutate(rng, seq, rate):
    s = seq.copy()
    m = rng.random(s.size) < rate
    s[m] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(m.sum()))]
    return s


def _make_requests(rng, genome, n_req, insert_frac=0.15):
    """(op, base, ranges) tuples; queries sample reads from the genome and
    from inserts issued before *or after* them, so order matters."""
    reqs = []
    pool = [genome]
    for _ in range(n_req):
        if rng.random() < insert_frac:
            parts, ranges, pos = [], [], int(rng.integers(0, 20))
            parts.append(random_dna(rng, pos))
            for _ in range(int(rng.integers(1, 5))):
                n = int(rng.integers(10, 20000))
                parts.append(random_dna(rng, n, b"ACGTACGTACGTACGTN"))
                ranges.append((pos, n))
                pos += n
            base = np.concatenate(parts)
            reqs.append((0, base, np.asarray(ranges, np.uint64)))
            pool.append(base)
        else:
            n_reads = int(rng.integers(1, 200))
            parts, ranges, pos = [], [], int(rng.integers(0, 40))
            parts.append(random_dna(rng, pos))
            for _ in range(n_reads):
                ln = int(rng.integers(20, 300))
                src = pool[int(rng.integers(0, len(pool)))] if rng.random() < 0.7 else None
                if src is not None and src.size > ln:
                    o = int(rng.integers(0, src.size - ln))
                    read = _mutate(rng, src[o:o + ln], 0.01)
                else:
                    read = random_dna(rng, ln)
                if rng.random() >= 0.3:  # otherwise adjacent to the previous read
                    g = int(rng.integers(1, 5))
                    parts.append(random_dna(rng, g))
                    pos += g
                parts.append(read)
                ranges.append((pos, ln))
                pos += ln
            base = np.concatenate(parts)
            reqs.append((1, base, np.asarray(ranges, np.uint64)))
        # Earlier queries may sample from inserts that come after them.
        if rng.random() < 0.1:
            future = random_dna(rng, 5000)
            pool.append(future)
            reqs.append((0, future, np.asarray([(0, 5000)], np.uint64)))
    return reqs


def _serial(sbf, genome, reqs, bits):
    """One request at a time, in order, through the ragged host API."""
    f = sbf.Filter(bits, **K31)
    f.insert_sequence(genome)
    outs = []
    for op, base, ranges in reqs:
        if op == 0:
            f.ragged_insert(base, ranges)
            outs.append(None)
        else:
            lo = int(ranges[0, 0])
            hi = int(ranges[-1, 0] + ranges[-1, 1])
            hits, _ = f.ragged_query(base, ranges)
            outs.append(hits[lo:max(lo, hi - 30)].copy())
    return outs, f.words_host()


def _served(sbf, genome, reqs, bits, **cfg):
    f = sbf.Filter(bits, **K31)
    f.insert_sequence(genome)
    srv = sbf.Server(f, staging_bytes=1 << 28, pinned_bytes=1 << 26, **cfg)
    tickets = [srv.submit(op, base, ranges) for op, base, ranges in reqs]
    outs = []
    for (op, _, _), t in zip(reqs, tickets):
        info, hits = srv.wait(t, timeout=60.0)
        assert info["status"] == 0 and info["latency_s"] >= 0
        outs.append(None if op == 0 else hits.copy())
    stats = srv.stats()
    srv.close()
    return outs, f.words_host(), stats


@pytest.mark.parametrize("cfg", [dict(), dict(use_graph=1, max_inflight=2),
                                 dict(max_batch_bytes=1 << 18, max_inflight=4)],
                         ids=["default", "graph", "small-batches"])
@pytest.mark.parametrize("expand", ["0", "1"], ids=["byte-download", "host-expand"])
def test_served_equals_serial(sbf, cuda, monkeypatch, cfg, expand):
    """Byte results (op 1) either come down as bytes or as bits that the
    completion thread expands; both equal the serial byte-download path."""
    rng = np.random.default_rng(17)
    genome = random_dna(rng, 400_000)
    reqs = _make_requests(rng, genome, 250)
    bits = 1 << 22
    monkeypatch.setenv("SBF_HOST_EXPAND", "0")
    want, want_words = _serial(sbf, genome, reqs, bits)
    monkeypatch.setenv("SBF_HOST_EXPAND", expand)
    got, words, stats = _served(sbf, genome, reqs, bits, **cfg)
    np.testing.assert_array_equal(words, want_words)
    for i, (w, g) in enumerate(zip(want, got)):
        if w is None:
            assert g is None
        else:
            np.testing.assert_array_equal(g, w, err_msg=f"request {i}")
    assert stats["requests"] == len(reqs)
    assert stats["p50_s"] <= stats["p99_s"] <= stats["p999_s"] <= stats["max_s"]
    if "max_batch_bytes" not in cfg:
        assert stats["mean_batch_requests"] > 1.0, "requests should have been coalesced"


def test_pinned_requests_match(sbf, cuda):
    """Requests whose sequences, ranges and outputs live in pinned memory take
    the direct-copy path; results match the serial pageable path."""
    torch = cuda
    rng = np.random.default_rng(23)
    genome = random_dna(rng, 300_000)
    reqs = [r for r in _make_requests(rng, genome, 60, insert_frac=0.0) if r[0] == 1]
    bits = 1 << 21
    want, _ = _serial(sbf, genome, reqs, bits)
    f = sbf.Filter(bits, **K31)
    f.insert_sequence(genome)
    srv = sbf.Server(f, staging_bytes=1 << 28, pinned_bytes=1 << 26)
    keep, tickets = [], []
    for _, base, ranges in reqs:
        pb = torch.from_numpy(base).pin_memory()
        pr = torch.from_numpy(ranges.view(np.int64)).pin_memory()
        span = int(ranges[-1, 0] + ranges[-1, 1] - ranges[0, 0])
        out = torch.zeros(max(span - 30, 1), dtype=torch.uint8).pin_memory()
        keep.append((pb, pr, out))
        tickets.append(srv.submit_raw(1, pb.data_ptr(), pr.data_ptr(), ranges.shape[0],
                                      out.data_ptr(), out.numel()))
    for t, w, (_, _, out) in zip(tickets, want, keep):
        info, _ = srv.wait(t, timeout=60.0)
        np.testing.assert_array_equal(out.numpy()[:info["windows"]], w)
    srv.close()


def test_one_request_per_launch_matches(sbf, cuda):
    rng = np.random.default_rng(3)
    genome = random_dna(rng, 200_000)
    reqs = _make_requests(rng, genome, 80)
    bits = 1 << 21
    want, want_words = _serial(sbf, genome, reqs, bits)
    got, words, stats = _served(sbf, genome, reqs, bits, max_batch_requests=1, max_inflight=1)
    np.testing.assert_array_equal(words, want_words)
    for w, g in zip(want, got):
        if w is not None:
            np.testing.assert_array_equal(g, w)
    assert stats["mean_batch_requests"] == 1.0


def test_concurrent_submitters_follow_ticket_order(sbf, cuda):
    rng = np.random.default_rng(8)
    genome = random_dna(rng, 300_000)
    reqs = _make_requests(rng, genome, 160)
    bits = 1 << 22
    f = sbf.Filter(bits, **K31)
    f.insert_sequence(genome)
    srv = sbf.Server(f, staging_bytes=1 << 28, pinned_bytes=1 << 26)
    order = []
    lock = threading.Lock()

    def worker(idx):
        for i in range(idx, len(reqs), 4):
            op, base, ranges = reqs[i]
            with lock:  # ticket order = the order recorded here
                t = srv.submit(op, base, ranges)
                order.append((t, i))

    ths = [threading.Thread(target=worker, args=(j,)) for j in range(4)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    order.sort()
    got = {}
    for t, i in order:
        _, hits = srv.wait(t, timeout=60.0)
        got[i] = None if hits is None else hits.copy()
    srv.close()
    seq = [reqs[i] for _, i in order]
    want, want_words = _serial(sbf, genome, seq, bits)
    np.testing.assert_array_equal(f.words_host(), want_words)
    for (_, i), w in zip(order, want):
        if w is not None:
            np.testing.assert_array_equal(got[i], w)


def test_server_rejects_bad_requests(sbf, cuda):
    f = sbf.Filter(1 << 20, **K31)
    srv = sbf.Server(f, staging_bytes=1 << 24, pinned_bytes=1 << 22, max_batch_bytes=1 << 20)
    seq = np.frombuffer(b"ACGT" * 100, np.uint8)
    with pytest.raises(sbf.SbfError):
        srv.submit(1, seq, [(0, 100)], out=np.zeros(10, np.uint8))  # output too small
    with pytest.raises(sbf.SbfError):
        srv.submit(1, seq, [(50, 10), (0, 10)])  # unordered
    big = np.zeros(2 << 20, np.uint8)
    with pytest.raises(sbf.SbfError):
        srv.submit(0, big, [(0, big.size)])  # above the batch cap
    t = srv.submit(1, seq, [(0, 400)])
    info, hits = srv.wait(t, timeout=30.0)
    assert info["windows"] == 370 and hits.size == 370 and not hits.any()
    srv.drain()
    srv.close()


def test_bit_packed_requests_match_bytes(sbf, cuda):
    """Op 2 returns the byte results packed one bit per window, in the same
    order relative to inserts (bit-packed and byte queries interleaved)."""
    rng = np.random.default_rng(31)
    genome = random_dna(rng, 300_000)
    reqs = _make_requests(rng, genome, 120)
    bits = 1 << 22
    want, want_words = _serial(sbf, genome, reqs, bits)
    f = sbf.Filter(bits, **K31)
    f.insert_sequence(genome)
    srv = sbf.Server(f, staging_bytes=1 << 28, pinned_bytes=1 << 26)
    ops = [op if op == 0 else (2 if i % 2 else 1) for i, (op, _, _) in enumerate(reqs)]
    tickets = [srv.submit(op, base, ranges) for op, (_, base, ranges) in zip(ops, reqs)]
    for op, t, w in zip(ops, tickets, want):
        _, hits = srv.wait(t, timeout=60.0)
        if op == 1:
            np.testing.assert_array_equal(hits, w)
        elif op == 2:
            b = np.packbits(w.astype(np.uint8), bitorder="little")
            b = np.concatenate([b, np.zeros(hits.size * 4 - b.size, np.uint8)])
            np.testing.assert_array_equal(hits, b.view(np.uint32))
    srv.close()
    np.testing.assert_array_equal(f.words_host(), want_words)


_VALID = np.zeros(256, bool)
_VALID[np.frombuffer(b"ACGTacgt", np.uint8)] = True


def _record_counts(base, ranges, span_hits, k=31):
    """Per-record (valid, positive) windows from a request's byte results."""
    lo = int(ranges[0, 0])
    out = np.zeros((ranges.shape[0], 2), np.uint64)
    for i, (off, ln) in enumerate(ranges.astype(np.int64)):
        if ln < k:
            continue
        bad = np.concatenate([[0], np.cumsum(~_VALID[base[off:off + ln]])])
        out[i, 0] = int(((bad[k:] - bad[:-k]) == 0).sum())
        out[i, 1] = int(span_hits[off - lo:off - lo + ln - k + 1].sum())
    return out


@pytest.mark.parametrize("cfg", [dict(), dict(use_graph=1, max_inflight=2)],
                         ids=["default", "graph"])
def test_count_requests_match_bytes(sbf, cuda, cfg):
    """Op 3 returns each record's valid and positive windows (counted in the
    query kernel's epilogue), interleaved with byte and bit-packed queries
    and inserts, equal to the counts of the serial byte results."""
    rng = np.random.default_rng(37)
    genome = random_dna(rng, 300_000)
    reqs = _make_requests(rng, genome, 150)
    bits = 1 << 22
    want, want_words = _serial(sbf, genome, reqs, bits)
    f = sbf.Filter(bits, **K31)
    f.insert_sequence(genome)
    srv = sbf.Server(f, staging_bytes=1 << 28, pinned_bytes=1 << 26, **cfg)
    ops = [op if op == 0 else (1, 2, 3)[i % 3] for i, (op, _, _) in enumerate(reqs)]
    tickets = [srv.submit(op, base, ranges) for op, (_, base, ranges) in zip(ops, reqs)]
    n_counts = 0
    for op, t, w, (_, base, ranges) in zip(ops, tickets, want, reqs):
        _, res = srv.wait(t, timeout=60.0)
        if op == 1:
            np.testing.assert_array_equal(res, w)
        elif op == 3:
            np.testing.assert_array_equal(res, _record_counts(base, ranges, w))
            n_counts += 1
    srv.close()
    assert n_counts > 20
    np.testing.assert_array_equal(f.words_host(), want_words)


def _dense_equivalent(base):
    """The bytes a 2-bit dense round trip gives: invalid bases (N) pack as
    code 3 and come back as G (dense_packed.hpp:36-50)."""
    s = base.copy()
    s[~_VALID[s]] = ord("G")
    return s


def _pack_bits(hits):
    b = np.packbits(hits.astype(np.uint8), bitorder="little")
    n_words = max((hits.size + 31) // 32, 1)
    b = np.concatenate([b, np.zeros(n_words * 4 - b.size, np.uint8)])
    return b.view(np.uint32)[:(hits.size + 31) // 32]


@pytest.mark.parametrize("cfg", [dict(), dict(use_graph=1, max_inflight=2),
                                 dict(max_batch_bytes=1 << 18, max_inflight=4)],
                         ids=["default", "graph", "small-batches"])
def test_dense_requests_match_serial(sbf, cuda, cfg):
    """Requests with 2-bit dense-packed bodies (op | 0x10), mixed with byte
    requests of every op, equal serial execution of the same bases."""
    rng = np.random.default_rng(43)
    genome = random_dna(rng, 300_000)
    reqs = [(op, _dense_equivalent(base), ranges)
            for op, base, ranges in _make_requests(rng, genome, 160)]
    bits = 1 << 22
    want, want_words = _serial(sbf, genome, reqs, bits)
    f = sbf.Filter(bits, **K31)
    f.insert_sequence(genome)
    srv = sbf.Server(f, staging_bytes=1 << 28, pinned_bytes=1 << 26, **cfg)
    ops, tickets = [], []
    for i, (op, base, ranges) in enumerate(reqs):
        q = op if op == 0 else (1, 2, 3)[i % 3]
        dense = i % 2 == 0
        body = sbf.pack_dense_sequence(base) if dense else base
        ops.append(q)
        tickets.append(srv.submit(q | (sbf.Server.DENSE if dense else 0), body, ranges))
    for i, (q, t, w, (_, base, ranges)) in enumerate(zip(ops, tickets, want, reqs)):
        info, res = srv.wait(t, timeout=60.0)
        assert info["status"] == 0
        if q == 1:
            np.testing.assert_array_equal(res, w, err_msg=f"request {i}")
        elif q == 2:
            np.testing.assert_array_equal(res, _pack_bits(w), err_msg=f"request {i}")
        elif q == 3:
            np.testing.assert_array_equal(res, _record_counts(base, ranges, w))
    srv.close()
    np.testing.assert_array_equal(f.words_host(), want_words)
