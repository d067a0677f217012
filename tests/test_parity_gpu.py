"""Bit-exact parity of the CUDA engine with the oracle (GPU).

Every case inserts the same seeded bytes into the engine (through the C ABI)
and into the oracle, then compares the full shard word array, and compares
every query byte.  Cases cover the tile/strip boundaries of the kernels
(8192-window tiles, 32-window strips), misaligned input and output pointers,
invalid bases, lower case, tiny filters (heavy shard collisions, so many runs
hit the same shard words through bulk OR-reductions), and the other compiled
configurations.
"""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

K31 = dict(k=31, s=28, m=16, hashes=4)


def _to_dev(torch, host: np.ndarray, offset: int = 0):
    """Copies `host` to a fresh device buffer starting `offset` bytes past a
    256-byte aligned allocation, so kernels see a misaligned pointer."""
    buf = torch.empty(host.size + offset + 16, dtype=torch.uint8, device="cuda")
    view = buf[offset:offset + host.size]
    view.copy_(torch.from_numpy(host))
    return view


def _engine_insert_query(sbf, torch, cfg, bits, ins, qry, in_off=0, out_off=0):
    f = sbf.Filter(bits, **cfg)
    d_ins = _to_dev(torch, ins, in_off)
    n = f.insert_sequence_async(d_ins)
    assert n == max(0, ins.size - cfg["k"] + 1)
    torch.cuda.synchronize()
    words = f.words_host()
    nq = f.kmer_count(qry.size)
    out_buf = torch.full((nq + out_off + 32,), 0xAB, dtype=torch.uint8, device="cuda")
    d_out = out_buf[out_off:out_off + max(nq, 1)]
    d_q = _to_dev(torch, qry, (in_off * 7) % 16)
    f.contains_sequence_async(d_q, d_out)
    torch.cuda.synchronize()
    hits = out_buf.cpu().numpy()
    # Bytes outside the output span must be untouched.
    assert (hits[:out_off] == 0xAB).all()
    assert (hits[out_off + nq:] == 0xAB).all()
    f.close()
    return words, hits[out_off:out_off + nq]


def _oracle_insert_query(oracle_mod, cfg, bits, ins, qry):
    o = oracle_mod.Oracle(**cfg)
    w = o.new_words(bits)
    o.insert(w, ins)
    return w, o.contains(w, qry)


@pytest.mark.parametrize("length", [0, 1, 30, 31, 32, 47, 48, 100, 4096 + 30, 4097 + 30,
                                    4096 * 3 + 29, 65536 + 13, 250_000])
def test_lengths_k31(sbf, cuda, oracle_mod, length):
    rng = np.random.default_rng(1000 + length)
    ins = random_dna(rng, length)
    qry = np.concatenate([ins[: length // 2], random_dna(rng, length)])
    bits = 1 << 16
    w_e, h_e = _engine_insert_query(sbf, cuda, K31, bits, ins, qry)
    w_o, h_o = _oracle_insert_query(oracle_mod, K31, bits, ins, qry)
    np.testing.assert_array_equal(w_e, w_o)
    np.testing.assert_array_equal(h_e, h_o)


@pytest.mark.parametrize("in_off,out_off", [(0, 0), (1, 0), (3, 5), (7, 15), (15, 1), (8, 8)])
def test_misaligned_pointers(sbf, cuda, oracle_mod, in_off, out_off):
    rng = np.random.default_rng(7 + in_off * 16 + out_off)
    ins = random_dna(rng, 3 * 4096 + 77)
    qry = np.concatenate([ins[100:5000], random_dna(rng, 9000)])
    bits = 1 << 18
    w_e, h_e = _engine_insert_query(sbf, cuda, K31, bits, ins, qry, in_off, out_off)
    w_o, h_o = _oracle_insert_query(oracle_mod, K31, bits, ins, qry)
    np.testing.assert_array_equal(w_e, w_o)
    np.testing.assert_array_equal(h_e, h_o)


@pytest.mark.parametrize("bits", [1, 256, 1 << 10, 1 << 14, 1 << 22, 1 << 28])
def test_filter_sizes(sbf, cuda, oracle_mod, bits):
    rng = np.random.default_rng(bits % 1000003)
    ins = random_dna(rng, 60_000)
    qry = np.concatenate([ins[:20_000], random_dna(rng, 40_000)])
    w_e, h_e = _engine_insert_query(sbf, cuda, K31, bits, ins, qry)
    w_o, h_o = _oracle_insert_query(oracle_mod, K31, bits, ins, qry)
    np.testing.assert_array_equal(w_e, w_o)
    np.testing.assert_array_equal(h_e, h_o)


def test_invalid_bases_and_case(sbf, cuda, oracle_mod):
    rng = np.random.default_rng(99)
    ins = random_dna(rng, 80_000, b"ACGTACGTACGTacgtNnRY-\n")
    # Long N runs and isolated Ns.
    ins[5000:5600] = ord("N")
    ins[40_000] = ord("N")
    qry = np.concatenate([ins[::-1].copy(), random_dna(rng, 30_000, b"ACGTN")])
    for bits in (1 << 12, 1 << 20):
        w_e, h_e = _engine_insert_query(sbf, cuda, K31, bits, ins, qry, 5, 3)
        w_o, h_o = _oracle_insert_query(oracle_mod, K31, bits, ins, qry)
        np.testing.assert_array_equal(w_e, w_o)
        np.testing.assert_array_equal(h_e, h_o)


def test_all_bytes(sbf, cuda, oracle_mod):
    """Every byte value appears; only A/C/G/T in either case is valid."""
    rng = np.random.default_rng(5)
    raw = rng.integers(0, 256, size=50_000, dtype=np.uint8)
    mix = random_dna(rng, 50_000, b"ACGTacgt")
    ins = np.where(rng.random(50_000) < 0.97, mix, raw).astype(np.uint8)
    qry = np.concatenate([ins, rng.integers(0, 256, size=10_000, dtype=np.uint8)])
    w_e, h_e = _engine_insert_query(sbf, cuda, K31, 1 << 16, ins, qry, 2, 9)
    w_o, h_o = _oracle_insert_query(oracle_mod, K31, 1 << 16, ins, qry)
    np.testing.assert_array_equal(w_e, w_o)
    np.testing.assert_array_equal(h_e, h_o)


def test_repeats_long_runs(sbf, cuda, oracle_mod):
    """Low-complexity input: very long super-k-mer runs and periodic repeats."""
    parts = [np.frombuffer(b"A" * 20_000, np.uint8), np.frombuffer(b"ACGT" * 5_000, np.uint8),
             np.frombuffer(b"AC" * 7_000, np.uint8)]
    rng = np.random.default_rng(3)
    unit = random_dna(rng, 173)
    parts.append(np.tile(unit, 100))
    ins = np.concatenate(parts)
    qry = np.concatenate([ins, random_dna(rng, 10_000)])
    w_e, h_e = _engine_insert_query(sbf, cuda, K31, 1 << 20, ins, qry)
    w_o, h_o = _oracle_insert_query(oracle_mod, K31, 1 << 20, ins, qry)
    np.testing.assert_array_equal(w_e, w_o)
    np.testing.assert_array_equal(h_e, h_o)


@pytest.mark.parametrize("cfg", [
    dict(k=31, s=30, m=16, hashes=4), dict(k=31, s=31, m=16, hashes=4),
    dict(k=31, s=28, m=16, hashes=8), dict(k=31, s=28, m=16, hashes=16),
    dict(k=21, s=19, m=11, hashes=4), dict(k=5, s=4, m=3, hashes=4), dict(k=3, s=2, m=2, hashes=4),
    dict(k=31, s=28, m=21, hashes=4), dict(k=31, s=30, m=21, hashes=4),
    dict(k=31, s=31, m=21, hashes=4),
])
def test_other_configs(sbf, cuda, oracle_mod, cfg):
    rng = np.random.default_rng(cfg["k"] * 100 + cfg["hashes"] + cfg["s"])
    ins = random_dna(rng, 30_000, b"ACGTACGTACGTN")
    qry = np.concatenate([ins[:10_000], random_dna(rng, 20_000)])
    for bits in (1 << 12, 1 << 20):
        w_e, h_e = _engine_insert_query(sbf, cuda, cfg, bits, ins, qry, 3, 7)
        w_o, h_o = _oracle_insert_query(oracle_mod, cfg, bits, ins, qry)
        np.testing.assert_array_equal(w_e, w_o)
        np.testing.assert_array_equal(h_e, h_o)


@pytest.mark.parametrize("num_symbols", [31, 32, 33, 63, 64, 65, 4096 + 30, 4096 * 2 + 31, 100_003])
def test_dense_packed(sbf, cuda, oracle_mod, num_symbols):
    torch = cuda
    rng = np.random.default_rng(num_symbols)
    seq = random_dna(rng, num_symbols, b"ACGTN")
    o = oracle_mod.Oracle(**K31)
    packed_o = o.pack_dense(seq)
    np.testing.assert_array_equal(sbf.pack_dense_sequence(seq), packed_o)
    d_seq = _to_dev(torch, seq, 3)
    d_words = torch.zeros(max(len(packed_o), 1) + 1, dtype=torch.int64, device="cuda")
    sbf.pack_dense_sequence_device(d_seq, num_symbols, d_words)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_words.cpu().numpy().view(np.uint64)[: len(packed_o)], packed_o)

    bits = 1 << 16
    f = sbf.Filter(bits, **K31)
    n = f.insert_dense_packed_async(d_words[: len(packed_o)], num_symbols)
    assert n == num_symbols - 30
    torch.cuda.synchronize()
    w_o = o.new_words(bits)
    o.insert_dense(w_o, packed_o, num_symbols)
    np.testing.assert_array_equal(f.words_host(), w_o)

    q = random_dna(rng, num_symbols, b"ACGT")
    q[: num_symbols // 2] = seq[: num_symbols // 2]
    qp = o.pack_dense(q)
    d_qp = torch.from_numpy(qp.view(np.int64)).cuda()
    d_out = torch.zeros(num_symbols, dtype=torch.uint8, device="cuda")
    f.contains_dense_packed_async(d_qp, num_symbols, d_out[5:])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_out[5:5 + num_symbols - 30].cpu().numpy(),
                                  o.contains_dense(w_o, qp, num_symbols))
    # Host dense variants.
    f.clear()
    assert f.insert_dense_packed(packed_o, num_symbols) == num_symbols - 30
    np.testing.assert_array_equal(f.words_host(), w_o)
    np.testing.assert_array_equal(f.contains_dense_packed(qp, num_symbols),
                                  o.contains_dense(w_o, qp, num_symbols))


@pytest.mark.parametrize("chunk", ["4096", "65536", None])
def test_host_pipeline(sbf, cuda, oracle_mod, monkeypatch, chunk):
    """Host-buffer APIs (chunked, double-buffered staging) equal the oracle,
    with pageable and pinned host memory."""
    torch = cuda
    if chunk:
        monkeypatch.setenv("SBF_HOST_CHUNK_BYTES", chunk)
    rng = np.random.default_rng(11)
    ins = random_dna(rng, 300_001, b"ACGTACGTN")
    qry = np.concatenate([ins[1000:150_000], random_dna(rng, 100_000)])
    bits = 1 << 20
    f = sbf.Filter(bits, **K31)
    assert f.insert_sequence(ins) == ins.size - 30
    w_o, h_o = _oracle_insert_query(oracle_mod, K31, bits, ins, qry)
    np.testing.assert_array_equal(f.words_host(), w_o)
    np.testing.assert_array_equal(f.contains_sequence(qry), h_o)
    # Pinned host buffers take the direct-copy path.
    pinned_in = torch.from_numpy(qry).pin_memory()
    np.testing.assert_array_equal(f.contains_sequence(pinned_in.numpy()), h_o)
    d_out = torch.zeros(h_o.size, dtype=torch.uint8, device="cuda")
    f.contains_sequence(qry, d_out=d_out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_out.cpu().numpy(), h_o)
    f.clear()
    assert f.insert_sequence(torch.from_numpy(ins).pin_memory().numpy()) == ins.size - 30
    np.testing.assert_array_equal(f.words_host(), w_o)


def test_reference_known_answers(sbf, cuda):
    """The reference's own GPU known answers (tests/test_bloom_filter.cu of
    tdortman/cuSBF) through the engine."""
    c5 = dict(k=5, s=4, m=3, hashes=4)
    f = sbf.Filter(1 << 12, **c5)
    seq = "ACGTNACGTACGTA"
    assert f.insert_sequence(seq) == 10
    assert list(f.contains_sequence(seq)) == [0, 0, 0, 0, 0, 1, 1, 1, 1, 1]  # :91-101

    f = sbf.Filter(1 << 12, **c5)  # :10-20 no false negatives
    seq = "ACGTACGTACGTACGT"
    assert f.insert_sequence(seq) == 12
    assert f.contains_sequence(seq).all()
    lf = f.load_factor()
    f.insert_sequence(seq)  # :103-115 idempotent
    assert f.load_factor() == lf
    f.clear()  # :154-163
    assert not f.contains_sequence(seq).any()

    f = sbf.Filter(1 << 12, **c5)  # :117-128 short inputs
    assert f.insert_sequence("ACGT") == 0
    assert f.contains_sequence("ACGT").size == 0

    f = sbf.Filter(1 << 12, **c5)  # :228-241 lower case
    f.insert_sequence("acgtacgtacgtacgt")
    assert f.contains_sequence("ACGTACGTACGTACGT").all()
    assert f.contains_sequence("acgtacgtacgtacgt").all()

    # :130-152 short sequence leaves the device output untouched.
    torch = cuda
    d_seq = torch.tensor(list(b"ACGT"), dtype=torch.uint8, device="cuda")
    d_out = torch.full((1,), 0xAB, dtype=torch.uint8, device="cuda")
    f.contains_sequence_async(d_seq, d_out)
    torch.cuda.synchronize()
    assert d_out.item() == 0xAB

    # :373-422 device record batch: separator windows read 0.
    f = sbf.Filter(1 << 14, **c5)
    r1, r2 = "ACGTACGTACGT", "TTGGAACCTTGG"
    f.insert_sequence(r1)
    f.insert_sequence(r2)
    hits = f.contains_sequence(r1 + "N" + r2)
    assert list(hits) == [1] * 8 + [0] * 5 + [1] * 8


def test_errors(sbf, cuda):
    # The reference's Config rules: a DNA k-mer fits 64 bits (k <= 32), and
    # a 31-symbol protein k-mer (5 bits a symbol) does not.
    with pytest.raises(sbf.SbfError) as e:
        sbf.Filter(1 << 10, k=33, s=9, m=5, hashes=4)
    assert e.value.category == "invalid_argument"
    with pytest.raises(sbf.SbfError) as e:
        sbf.Filter(1 << 10, alphabet=2)
    assert e.value.category == "invalid_argument"
    torch = cuda
    f = sbf.Filter(1 << 12)
    d = torch.zeros(100, dtype=torch.uint8, device="cuda")
    with pytest.raises(sbf.SbfError) as e:
        f.contains_sequence_async(d, d[:10])
    assert e.value.category == "invalid_argument"
    with pytest.raises(sbf.SbfError):
        f.insert_dense_packed_async(torch.zeros(1, dtype=torch.int64, device="cuda"), 100)
