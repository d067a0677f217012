"""Configurations without a specialised tile kernel run on the generic
kernels (sbf_generic.cu): any k, s, m and hash count of the reference's
Config, and the protein and DNA-triplet alphabets.  Checked bit for bit
against the oracle (and against the reference's own arithmetic where
oracle/_ref holds that configuration) through the sequence, bit-packed,
dense-packed, host-pipeline, ragged, per-record-count, record-batch and FASTX
entry points."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _generic_kernels(monkeypatch):
    """DNA configurations would otherwise run tile kernels compiled at run
    time (tests/test_jit_gpu.py); here they exercise the generic kernels."""
    monkeypatch.setenv("SBF_JIT", "0")

DNA, TRIPLET, PROTEIN = 0, 1, 2
AMINO = b"ACDEFGHIKLMNPQRSTVWYacdefghiklmnpqrstvwyBXZ"

CONFIGS = [
    dict(k=25, s=22, m=13, hashes=4, alphabet=DNA),
    dict(k=17, s=15, m=9, hashes=8, alphabet=DNA),
    dict(k=32, s=32, m=32, hashes=12, alphabet=DNA),
    dict(k=1, s=1, m=1, hashes=16, alphabet=DNA),
    dict(k=5, s=4, m=3, hashes=4, alphabet=PROTEIN),
    dict(k=12, s=10, m=6, hashes=8, alphabet=PROTEIN),
    dict(k=3, s=2, m=2, hashes=4, alphabet=TRIPLET),
    dict(k=10, s=8, m=5, hashes=16, alphabet=TRIPLET),
]
IDS = ["dna25", "dna17h8", "dna32h12", "dna1h16", "prot5", "prot12h8", "trip3", "trip10h16"]
WIDTH = {DNA: 1, PROTEIN: 1, TRIPLET: 3}


def _seq(rng, cfg, n_sym, dirty=True):
    if cfg["alphabet"] == PROTEIN:
        a = np.frombuffer(AMINO + (b"*1 -" if dirty else b""), np.uint8)
        return a[rng.integers(0, a.size, n_sym * WIDTH[PROTEIN])]
    alpha = b"ACGTACGTACGTACGTacgtN" if dirty else b"ACGT"
    return random_dna(rng, n_sym * WIDTH[cfg["alphabet"]] + int(rng.integers(0, 3)), alpha)


def _oracle(oracle_mod, cfg):
    return oracle_mod.Oracle(**cfg)


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_sequence_paths_match_oracle(sbf, cuda, oracle_mod, monkeypatch, cfg):
    torch = cuda
    rng = np.random.default_rng(cfg["k"] * 7 + cfg["hashes"] + cfg["alphabet"])
    bits = 1 << 16
    o = _oracle(oracle_mod, cfg)
    ins = _seq(rng, cfg, 40_000)
    qry = np.concatenate([ins[: 9000 * WIDTH[cfg["alphabet"]]], _seq(rng, cfg, 9000)])
    w = o.new_words(bits)
    o.insert(w, ins)
    want = o.contains(w, qry)
    # host pipeline with small chunks (chunk boundaries inside symbols for triplets)
    monkeypatch.setenv("SBF_HOST_CHUNK_BYTES", "4099")
    f = sbf.Filter(bits, **cfg)
    f.insert_sequence(ins)
    np.testing.assert_array_equal(f.words_host(), w)
    np.testing.assert_array_equal(f.contains_sequence(qry), want)
    assert f.kmer_count(qry.size) == want.size
    assert want.any() and not want.all()
    # device-resident and bit-packed
    g = sbf.Filter(bits, **cfg)
    d_ins = torch.from_numpy(ins.copy()).cuda()
    g.insert_sequence_async(d_ins)
    d_q = torch.from_numpy(qry.copy()).cuda()
    out = torch.full((want.size + 5,), 9, dtype=torch.uint8, device="cuda")
    g.contains_sequence_async(d_q, out[1:1 + want.size])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(g.words_host(), w)
    np.testing.assert_array_equal(out[1:1 + want.size].cpu().numpy(), want)
    packed = g.contains_sequence_bits(qry)
    expect = np.packbits(want, bitorder="little")
    expect = np.concatenate([expect, np.zeros(packed.size * 4 - expect.size, np.uint8)])
    np.testing.assert_array_equal(packed.view(np.uint8), expect)


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_dense_paths_match_oracle(sbf, cuda, oracle_mod, monkeypatch, cfg):
    torch = cuda
    rng = np.random.default_rng(cfg["k"] + 3 * cfg["hashes"] + cfg["alphabet"])
    bits = 1 << 15
    o = _oracle(oracle_mod, cfg)
    seq = _seq(rng, cfg, 30_000)
    n_sym = seq.size // WIDTH[cfg["alphabet"]]
    packed = sbf.pack_dense_sequence(seq, alphabet=cfg["alphabet"])
    np.testing.assert_array_equal(packed, o.pack_dense(seq))
    assert packed.size == sbf.Filter.dense_packed_word_count(n_sym, cfg["alphabet"])
    d_seq = torch.from_numpy(seq.copy()).cuda()
    d_words = torch.zeros(packed.size, dtype=torch.int64, device="cuda")
    sbf.pack_dense_sequence_device(d_seq, n_sym, d_words, alphabet=cfg["alphabet"])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_words.cpu().numpy().view(np.uint64), packed)
    w = o.new_words(bits)
    o.insert_dense(w, packed[: packed.size // 2], (packed.size // 2) * (64 // _bits(cfg)))
    want = o.contains_dense(w, packed, n_sym)
    monkeypatch.setenv("SBF_HOST_CHUNK_BYTES", "4096")
    f = sbf.Filter(bits, **cfg)
    f.insert_dense_packed(packed[: packed.size // 2], (packed.size // 2) * (64 // _bits(cfg)))
    np.testing.assert_array_equal(f.words_host(), w)
    np.testing.assert_array_equal(f.contains_dense_packed(packed, n_sym), want)
    assert want.any()


def _bits(cfg):
    return {DNA: 2, PROTEIN: 5, TRIPLET: 6}[cfg["alphabet"]]


@pytest.mark.parametrize("cfg", [c for c in CONFIGS if c["alphabet"] != TRIPLET],
                         ids=[i for i, c in zip(IDS, CONFIGS) if c["alphabet"] != TRIPLET])
def test_record_paths_match_oracle(sbf, cuda, oracle_mod, cfg):
    """Ragged batches, fused per-record counts, host record batches and FASTA
    input for one-byte alphabets, against the oracle run record by record."""
    torch = cuda
    rng = np.random.default_rng(cfg["k"] * 5 + cfg["alphabet"])
    o = _oracle(oracle_mod, cfg)
    k = cfg["k"]
    parts, ranges, pos = [], [], 0
    for i in range(300):
        if rng.random() < 0.3:
            g = _seq(rng, cfg, int(rng.integers(1, 9)))
            parts.append(g)
            pos += g.size
        n = int(rng.integers(0, 400)) if i % 10 else 0
        r = _seq(rng, cfg, n)[:n]
        parts.append(r)
        ranges.append((pos, r.size))
        pos += r.size
    seq = np.concatenate(parts)
    bits = 1 << 16
    f = sbf.Filter(bits, **cfg)
    rep = f.ragged_insert(seq, ranges[::2])
    w = o.new_words(bits)
    for off, n in ranges[::2]:
        o.insert(w, seq[off:off + n])
    np.testing.assert_array_equal(f.words_host(), w)
    hits, qrep = f.ragged_query(seq, ranges)
    valid = np.zeros(len(ranges), np.uint64)
    posv = np.zeros(len(ranges), np.uint64)
    for i, (off, n) in enumerate(ranges):
        if n < k:
            assert not hits[off:off + max(n - k + 1, 0)].any()
            continue
        want = o.contains(w, seq[off:off + n])
        np.testing.assert_array_equal(hits[off:off + n - k + 1], want)
        shards, ok = o.window_shards(seq[off:off + n], f.num_shards())
        valid[i], posv[i] = int(ok.sum()), int(want.sum())
    assert qrep.queried_kmers == int(valid.sum()) and qrep.positive_kmers == int(posv.sum())
    assert rep.inserted_kmers == int(valid[::2].sum())
    d_seq = torch.from_numpy(seq.copy()).cuda()
    d_rng = torch.from_numpy(np.asarray(ranges, np.uint64).view(np.int64).reshape(-1, 2)).cuda()
    rv = torch.zeros(len(ranges), dtype=torch.int64, device="cuda")
    rp = torch.zeros(len(ranges), dtype=torch.int64, device="cuda")
    f.ragged_contains_counts_async(d_seq, d_rng, rv, rp)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(rv.cpu().numpy().astype(np.uint64), valid)
    np.testing.assert_array_equal(rp.cpu().numpy().astype(np.uint64), posv)
    # host record batch: per-record counts and hits in the normalised layout
    recs = []
    qb = f.query_record_batch(seq, ranges, consume=recs.append)
    assert [r["positive_kmers"] for r in recs] == [int(x) for x in posv]
    assert [r["queried_kmers"] for r in recs] == [int(x) for x in valid]
    assert qb.positive_kmers == int(posv.sum())
    # FASTA records through the FASTX entry point
    fasta = b"".join(b">r%d\n" % i + seq[off:off + n].tobytes() + b"\n"
                     for i, (off, n) in enumerate(ranges))
    fq = f.query_fastx(fasta)
    assert fq.records_queried == len(ranges)
    assert fq.positive_kmers == int(posv.sum()) and fq.queried_kmers == int(valid.sum())


PROT = dict(k=5, s=4, m=3, hashes=4, alphabet=PROTEIN)   # ProteinTestConfig
TRIP = dict(k=3, s=2, m=2, hashes=4, alphabet=TRIPLET)   # TripletTestConfig


def test_reference_alphabet_known_answers(sbf, cuda):
    """The reference's alphabet tests (tests/test_bloom_filter.cu:73-90,
    243-338 of tdortman/cuSBF), restated."""
    f = sbf.Filter(1 << 14, **PROT)
    s = b"ACDEFGHIKLMNPQRSTVWYACDEF"
    packed = sbf.pack_dense_sequence(s, alphabet=PROTEIN)
    assert f.insert_dense_packed(packed, len(s)) == len(s) - 4
    hits = f.contains_dense_packed(packed, len(s))
    assert hits.size == len(s) - 4 and hits.all()
    np.testing.assert_array_equal(hits, f.contains_sequence(s))
    f = sbf.Filter(1 << 12, **PROT)
    s = b"ABCDEFGHIJKLMNOPQRSTUVWXYZ"
    assert f.insert_sequence(s) == len(s) - 4 and f.contains_sequence(s).all()
    f = sbf.Filter(1 << 12, **PROT)
    f.insert_sequence(s.lower())
    assert f.contains_sequence(s).all() and f.contains_sequence(s.lower()).all()
    f = sbf.Filter(1 << 12, **PROT)
    s = b"ACDE*ACDEFGHI"
    assert f.insert_sequence(s) == 9
    assert list(f.contains_sequence(s)) == [0, 0, 0, 0, 0, 1, 1, 1, 1]
    f = sbf.Filter(1 << 12, **TRIP)
    s = b"ACGTACGTTAAACCCGGGTTT"
    assert f.insert_sequence(s) == len(s) // 3 - 2 and f.contains_sequence(s).all()
    f = sbf.Filter(1 << 12, **TRIP)
    f.insert_sequence(s.lower())
    assert f.contains_sequence(s).all() and f.contains_sequence(s.lower()).all()
    f = sbf.Filter(1 << 12, **TRIP)
    s = b"ACGTACNNNGGGTTTAAA"
    assert f.insert_sequence(s) == 4
    assert list(f.contains_sequence(s)) == [0, 0, 0, 1]
    f = sbf.Filter(1 << 12, **TRIP)
    s = b"ACGTACGTTAAACCCGGGTTTAA"
    assert f.insert_sequence(s) == 5
    hits = f.contains_sequence(s)
    assert hits.size == 5 and hits.all()


def test_triplet_record_paths_match_oracle(sbf, cuda, oracle_mod):
    """Triplet record batches (ranges on symbol boundaries) and FASTA records
    of any length (each padded to a symbol boundary by normalisation)."""
    torch = cuda
    cfg = dict(k=6, s=5, m=3, hashes=8, alphabet=TRIPLET)
    rng = np.random.default_rng(41)
    o = oracle_mod.Oracle(**cfg)
    parts, ranges, pos = [], [], 0
    for i in range(200):
        n = 3 * int(rng.integers(0, 60))
        g = 3 * int(rng.integers(0, 3))
        parts.append(random_dna(rng, g + n, b"ACGTACGTACGTN"))
        ranges.append((pos + g, n))
        pos += g + n
    seq = np.concatenate(parts)
    bits = 1 << 16
    f = sbf.Filter(bits, **cfg)
    ins = f.insert_record_batch(seq, ranges[::2])
    w = o.new_words(bits)
    for off, n in ranges[::2]:
        o.insert(w, seq[off:off + n])
    np.testing.assert_array_equal(f.words_host(), w)
    recs = []
    rep = f.query_record_batch(seq, ranges, consume=recs.append)
    total = 0
    for (off, n), r in zip(ranges, recs):
        want = o.contains(w, seq[off:off + n])
        np.testing.assert_array_equal(r["hits"], want)
        assert r["positive_kmers"] == int(want.sum())
        total += int(want.sum())
    assert rep.positive_kmers == total
    assert ins.inserted_kmers == sum(int(o.window_shards(seq[a:a + n], 4)[1].sum())
                                     for a, n in ranges[::2])
    # the device record batch over the normalised sequence
    norm, nrecs = sbf.normalize_record_batch(cfg["k"], seq, ranges, alphabet=TRIPLET)
    layout, n_hits = sbf.query_layout(cfg["k"], nrecs, alphabet=TRIPLET)
    d_norm = torch.from_numpy(norm.copy()).cuda()
    d_out = torch.zeros(n_hits, dtype=torch.uint8, device="cuda")
    nranges = [(lr.hit_offset * 3, lr.size) for lr in layout]
    f.contains_record_batch_async(d_norm, nranges, d_out)
    torch.cuda.synchronize()
    h = d_out.cpu().numpy()
    for lr, r in zip(layout, recs):
        np.testing.assert_array_equal(h[lr.hit_offset:lr.hit_offset + lr.hit_count], r["hits"])
    # FASTA records of unaligned lengths: trailing partial symbols ignored
    fasta = b"".join(b">r%d\n" % i + random_dna(rng, int(rng.integers(0, 200))).tobytes() + b"\n"
                     for i in range(100))
    g = sbf.Filter(bits, **cfg)
    frep = g.insert_fastx(fasta)
    w2 = o.new_words(bits)
    lines = fasta.split(b"\n")
    want_kmers = 0
    for ln in lines[1::2]:
        a = np.frombuffer(ln, np.uint8)
        if a.size:
            o.insert(w2, a)
            want_kmers += int(o.window_shards(a, 4)[1].sum())
    np.testing.assert_array_equal(g.words_host(), w2)
    assert frep.records_indexed == 100 and frep.inserted_kmers == want_kmers


def test_triplets_reject_pipeline_paths(sbf, cuda):
    f = sbf.Filter(1 << 14, **TRIP)
    seq = np.frombuffer(b"ACGTACGTACGTACGTACGT" * 9, np.uint8)
    with pytest.raises(sbf.SbfError):
        f.ragged_insert(seq, [(0, 60)])
    with pytest.raises(sbf.SbfError):
        sbf.Server(f)
    with pytest.raises(sbf.SbfError):
        f.query_record_batch(seq, [(1, 60)])  # not on a symbol boundary
    assert f.insert_sequence(seq) == seq.size // 3 - 2


def test_reference_arithmetic_agrees(sbf, cuda, oracle_mod):
    """The configurations oracle/_ref builds from the reference's own headers
    (protein <5,4,3,4>, triplets <3,2,2,4>) against the generic kernels."""
    if not oracle_mod.RefCpu.available():
        pytest.skip("oracle/_ref is not built")
    rng = np.random.default_rng(3)
    for cfg in (dict(k=5, s=4, m=3, hashes=4, alphabet=PROTEIN),
                dict(k=3, s=2, m=2, hashes=4, alphabet=TRIPLET)):
        ref = oracle_mod.RefCpu(**cfg)
        seq = _seq(rng, cfg, 20_000)
        bits = 1 << 14
        w = ref_words = np.zeros(oracle_mod.num_shards(bits) * 4, np.uint64)
        ref.insert(ref_words, seq[: seq.size // 2])
        f = sbf.Filter(bits, **cfg)
        f.insert_sequence(seq[: seq.size // 2])
        np.testing.assert_array_equal(f.words_host(), w)
        np.testing.assert_array_equal(f.contains_sequence(seq), ref.contains(w, seq))
