"""FASTX insert/query on the GPU: the reference's tests/test_fastx.cu cases
(Config<5,4,3,4>) and parity of chunked FASTX queries with the oracle."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu
C5 = dict(k=5, s=4, m=3, hashes=4)
K31 = dict(k=31, s=28, m=16, hashes=4)


def test_wrapped_fasta_insert(sbf, cuda, tmp_path):
    # test_fastx.cu:23-41
    f = sbf.Filter(1 << 12, **C5)
    p = tmp_path / "w.fa"
    p.write_text(">wrapped\nACGT\nACGT\nACGT\n")
    rep = f.insert_fastx_file(p)
    assert (rep.records_indexed, rep.indexed_bases, rep.inserted_kmers) == (1, 12, 8)
    assert f.contains_sequence("ACGTACGTACGT").all()


def test_fastq_crlf_query_records_and_detailed(sbf, cuda, tmp_path):
    # test_fastx.cu:43-113, :325-358
    f = sbf.Filter(1 << 12, **C5)
    f.insert_sequence("ACGTACGTACGT")
    p = tmp_path / "w.fq"
    p.write_bytes(b"@wrapped\r\nACGTAC\r\nGTACGT\r\n+\r\nIIIIII\r\nIIIIII\r\n")
    rep = f.query_fastx_file(p)
    assert (rep.records_queried, rep.queried_bases, rep.queried_kmers, rep.positive_kmers) == (1, 12, 8, 8)
    summary, recs = f.query_fastx_file_detailed(p)
    assert summary.positive_kmers == 8 and len(recs) == 1
    r = recs[0]
    assert (r["record_index"], r["header"], r["sequence"]) == (0, "wrapped", b"ACGTACGTACGT")
    assert r["hits"].size == 8 and r["hits"].all()


def test_no_cross_record_kmers(sbf, cuda):
    # test_fastx.cu:114-141
    f = sbf.Filter(1 << 14, **C5)
    f.insert_sequence("ACGTACGT")
    f.insert_sequence("TGCATGCA")
    rep = f.query_fastx(">first\nACGT\nACGT\n>second\nTGCA\nTGCA\n")
    assert (rep.records_queried, rep.queried_bases) == (2, 16)
    assert rep.queried_kmers == 8 and rep.positive_kmers == 8


def test_reports_only_valid_kmers(sbf, cuda):
    # test_fastx.cu:306-323
    f = sbf.Filter(1 << 12, **C5)
    ins = f.insert_fastx(">with-invalid\nACGTNACGTACGTA\n")
    assert (ins.records_indexed, ins.indexed_bases, ins.inserted_kmers) == (1, 14, 5)
    q = f.query_fastx(">with-invalid\nACGTNACGTACGTA\n")
    assert (q.records_queried, q.queried_bases, q.queried_kmers, q.positive_kmers) == (1, 14, 5, 5)


@pytest.mark.parametrize("fill", [0.0, 0.7])
def test_forced_chunk_flush(sbf, cuda, tmp_path, fill):
    # test_fastx.cu:576-666
    f = sbf.Filter(1 << 12, **C5)
    p = tmp_path / "three.fa"
    p.write_text(">first\nACGTACGT\n>second\nACGTNACGTACGTA\n>third\nTGCATGCA\n")
    ins = f.insert_fastx_file(p, fill)
    agg = f.query_fastx_file(p, fill)
    streamed = []
    s2 = f.query_fastx_file_records(p, streamed.append, fill)
    summary, detailed = f.query_fastx_file_detailed(p, fill)
    assert (ins.records_indexed, ins.indexed_bases, ins.inserted_kmers) == (3, 30, 4 + 5 + 4)
    for r in (agg, s2, summary):
        assert (r.records_queried, r.queried_bases, r.queried_kmers, r.positive_kmers) == (3, 30, 13, 13)
    for recs in (streamed, detailed):
        assert [r["header"] for r in recs] == ["first", "second", "third"]
        assert [r["record_index"] for r in recs] == [0, 1, 2]
        assert recs[1]["hits"].tolist() == [0, 0, 0, 0, 0, 1, 1, 1, 1, 1]
        assert recs[0]["hits"].all() and recs[2]["hits"].all()


def test_explicit_stream_equivalence(sbf, cuda, tmp_path):
    # test_fastx.cu:667-707
    torch = cuda
    f = sbf.Filter(1 << 12, **C5)
    p = tmp_path / "three.fa"
    p.write_text(">first\nACGTACGT\n>second\nACGTNACGTACGTA\n>third\nTGCATGCA\n")
    f.insert_fastx_file(p, 0.0)
    a = f.query_fastx_file_detailed(p, 0.0)
    s = torch.cuda.Stream()
    b = f.query_fastx_file_detailed(p, 0.0, stream=s)
    assert a[0].positive_kmers == b[0].positive_kmers
    for x, y in zip(a[1], b[1]):
        assert x["header"] == y["header"] and (x["hits"] == y["hits"]).all()


def test_malformed_fastq_query(sbf, cuda, tmp_path):
    # test_fastx.cu:708-727
    f = sbf.Filter(1 << 12, **C5)
    p = tmp_path / "broken.fq"
    p.write_text("@broken\nACGTACGT\n+\nIIIIIII\n")
    with pytest.raises(sbf.SbfError) as e:
        f.query_fastx_file(p)
    assert e.value.category == "fastx_parse" and e.value.location[1:] == (4, 8)


def test_callback_abort_keeps_filter_usable(sbf, cuda):
    # test_fastx.cu:728-826
    f = sbf.Filter(1 << 12, **C5)
    for s in ("ACGTACGTACGT", "TGCATGCA", "GGGAAAACCC"):
        f.insert_sequence(s)
    text = ">seqA\nACGTACGTACGT\n>seqB\nTGCATGCA\n>seqC\nGGGAAAACCC\n"
    seen = []

    class Stop(Exception):
        pass

    def consume(r):
        seen.append(r["header"])
        if len(seen) == 2:
            raise Stop()
    with pytest.raises(Stop):
        f.query_fastx_records(text, consume, 0.0)
    assert seen == ["seqA", "seqB"]
    summary, recs = f.query_fastx_detailed(text)
    assert [r["header"] for r in recs] == ["seqA", "seqB", "seqC"]
    assert summary.positive_kmers == summary.queried_kmers == 8 + 4 + 6


@pytest.mark.parametrize("fill", [0.0, 0.7])
def test_fastx_parity_k31(sbf, cuda, oracle_mod, fill, tmp_path):
    """Reads queried through the FASTX path equal the oracle per record."""
    rng = np.random.default_rng(77)
    genome = random_dna(rng, 200_000, b"ACGTACGTN")
    reads = []
    for i in range(400):
        n = int(rng.integers(20, 400))
        if rng.random() < 0.6:
            p0 = int(rng.integers(0, genome.size - n))
            reads.append(genome[p0:p0 + n].copy())
        else:
            reads.append(random_dna(rng, n))
    fq = b"".join(b"@r%d\n" % i + r.tobytes() + b"\n+\n" + b"I" * r.size + b"\n"
                  for i, r in enumerate(reads))
    p = tmp_path / "reads.fq"
    p.write_bytes(fq)
    bits = 1 << 20
    f = sbf.Filter(bits, **K31)
    f.insert_fastx(b">g\n" + genome.tobytes() + b"\n", fill)
    o = oracle_mod.Oracle(**K31)
    w = o.new_words(bits)
    o.insert(w, genome)
    np.testing.assert_array_equal(f.words_host(), w)
    summary, recs = f.query_fastx_file_detailed(p, fill)
    assert len(recs) == len(reads)
    tot = 0
    for r, seq in zip(recs, reads):
        want = o.contains(w, seq)
        np.testing.assert_array_equal(r["hits"], want)
        assert r["positive_kmers"] == int(want.sum())
        tot += int(want.sum())
    assert summary.positive_kmers == tot
