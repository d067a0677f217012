"""FASTA parsed on the GPU gives exactly the host parser's results: reports,
filter words and per-record views, across block boundaries (tiny blocks),
wrapped and CRLF lines, blank lines, empty records, records longer than a
block (the block grows), gzip input, missing final newlines and a consumer
that aborts."""
import gzip

import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu
K31 = dict(k=31, s=28, m=16, hashes=4)


def _wrap(seq, width):
    if width <= 0:
        return seq + b"\n"
    return b"".join(seq[i:i + width] + b"\n" for i in range(0, len(seq), width)) or b"\n"


def _fasta(rng, genome, n, lo=0, hi=3000, width=60, extra=b""):
    out = []
    for i in range(n):
        ln = int(rng.integers(lo, hi))
        o = int(rng.integers(0, genome.size - ln))
        out.append(b">c%d some description\n" % i + extra + _wrap(genome[o:o + ln].tobytes(), width))
    return b"".join(out)


def _run(sbf, monkeypatch, parser, block, data_or_path, genome, query=True, as_file=False):
    monkeypatch.setenv("SBF_FASTX_PARSER", parser)
    if block:
        monkeypatch.setenv("SBF_FASTQ_BLOCK_BYTES", str(block))
    else:
        monkeypatch.delenv("SBF_FASTQ_BLOCK_BYTES", raising=False)
    f = sbf.Filter(1 << 22, **K31)
    f.insert_sequence(genome)
    recs = []
    if query:
        if as_file:
            rep = f.query_fastx_file(data_or_path, consume=recs.append)
        else:
            rep = f.query_fastx(data_or_path, consume=recs.append)
    else:
        rep = f.insert_fastx_file(data_or_path) if as_file else f.insert_fastx(data_or_path)
    return rep.as_dict(), f.words_host(), recs


def _same(a, b):
    ra, wa, la = a
    rb, wb, lb = b
    assert ra == rb
    np.testing.assert_array_equal(wa, wb)
    assert len(la) == len(lb)
    for x, y in zip(la, lb):
        for key in ("record_index", "header", "sequence", "queried_bases", "queried_kmers",
                    "positive_kmers"):
            assert x[key] == y[key], key
        np.testing.assert_array_equal(x["hits"], y["hits"])


@pytest.mark.parametrize("block", [4096, 5000, 65536, 0])
@pytest.mark.parametrize("width", [60, 0])
@pytest.mark.parametrize("crlf", [False, True])
def test_query_matches_host_parser(sbf, cuda, monkeypatch, block, width, crlf):
    rng = np.random.default_rng(block + 3 * width + crlf)
    genome = random_dna(rng, 200_000)
    data = _fasta(rng, genome, 150, width=width)
    data += _fasta(rng, random_dna(rng, 50_000), 50, hi=500, width=width)
    if crlf:
        data = data.replace(b"\n", b"\r\n")
    dev = _run(sbf, monkeypatch, "device", block, data, genome)
    host = _run(sbf, monkeypatch, "host", 0, data, genome)
    _same(dev, host)
    assert dev[0]["records_queried"] == 200
    assert dev[0]["positive_kmers"] > 0


@pytest.mark.parametrize("block", [4096, 0])
def test_insert_matches_host_parser(sbf, cuda, monkeypatch, tmp_path, block):
    rng = np.random.default_rng(5)
    genome = random_dna(rng, 300_000, b"ACGTACGTACGTacgtN")
    data = _fasta(rng, genome, 120, hi=20_000, width=80)
    p = tmp_path / "in.fa.gz"
    p.write_bytes(gzip.compress(data))
    seed = random_dna(rng, 1000)
    dev = _run(sbf, monkeypatch, "device", block, str(p), seed, query=False, as_file=True)
    host = _run(sbf, monkeypatch, "host", 0, str(p), seed, query=False, as_file=True)
    _same(dev, host)
    assert dev[0]["records_indexed"] == 120


@pytest.mark.parametrize("kind", ["blank-lines", "empty-records", "bare-header", "at-lines",
                                  "no-final-newline", "cr-only-lines", "single-record"])
def test_irregular_layouts(sbf, cuda, monkeypatch, kind):
    rng = np.random.default_rng(23)
    genome = random_dna(rng, 100_000)
    if kind == "blank-lines":
        data = _fasta(rng, genome, 40, width=70, extra=b"\n") + b"\n\n"
    elif kind == "empty-records":
        data = b">a\n>b\n" + _fasta(rng, genome, 30) + b">z\n"
    elif kind == "bare-header":
        data = b">\n" + genome[:3000].tobytes() + b"\n>\r\n" + genome[5000:5100].tobytes() + b"\n"
    elif kind == "at-lines":
        data = _fasta(rng, genome, 20, extra=b"@not a header\n+\n")
    elif kind == "no-final-newline":
        data = _fasta(rng, genome, 25) + b">end\n" + genome[:777].tobytes()
    elif kind == "cr-only-lines":
        data = _fasta(rng, genome, 25, extra=b"\r\n").replace(b"\n", b"\r\n")
    else:
        data = b">chr\n" + _wrap(genome.tobytes(), 61)
    for block in (4096, 0):
        dev = _run(sbf, monkeypatch, "device", block, data, genome)
        host = _run(sbf, monkeypatch, "host", 0, data, genome)
        _same(dev, host)


def test_record_longer_than_block(sbf, cuda, monkeypatch, tmp_path):
    # A 1 Mbp record through a 4 KiB block: the block doubles until the
    # record and the next header fit.
    rng = np.random.default_rng(29)
    genome = random_dna(rng, 1_000_000)
    data = (b">big\n" + _wrap(genome.tobytes(), 60) + _fasta(rng, genome, 10)
            + b">big2\n" + _wrap(genome[:200_000].tobytes(), 0))
    dev = _run(sbf, monkeypatch, "device", 4096, data, genome)
    host = _run(sbf, monkeypatch, "host", 0, data, genome)
    _same(dev, host)
    assert dev[0]["positive_kmers"] == dev[0]["queried_kmers"]
    p = tmp_path / "big.fa"
    p.write_bytes(data)
    seed = random_dna(rng, 100)
    dev = _run(sbf, monkeypatch, "device", 4096, str(p), seed, query=False, as_file=True)
    host = _run(sbf, monkeypatch, "host", 0, str(p), seed, query=False, as_file=True)
    _same(dev, host)


def test_insert_then_query_round_trip(sbf, cuda, monkeypatch):
    # Every k-mer of an inserted FASTA is found again when the same FASTA is
    # queried (no false negatives through the device parser).
    monkeypatch.setenv("SBF_FASTQ_BLOCK_BYTES", "8192")
    rng = np.random.default_rng(31)
    genome = random_dna(rng, 400_000)
    data = _fasta(rng, genome, 200, hi=5000, width=60)
    f = sbf.Filter(1 << 22, **K31)
    ins = f.insert_fastx(data)
    q = f.query_fastx(data)
    assert ins.records_indexed == q.records_queried == 200
    assert q.queried_kmers == ins.inserted_kmers
    assert q.positive_kmers == q.queried_kmers


def test_abort_from_consumer(sbf, cuda, monkeypatch):
    monkeypatch.setenv("SBF_FASTQ_BLOCK_BYTES", "4096")
    rng = np.random.default_rng(37)
    genome = random_dna(rng, 50_000)
    data = _fasta(rng, genome, 300, hi=400)
    f = sbf.Filter(1 << 20, **K31)
    seen = []

    def consume(r):
        seen.append(r["record_index"])
        if len(seen) == 120:
            raise RuntimeError("stop")

    with pytest.raises(RuntimeError):
        f.query_fastx(data, consume=consume)
    assert seen == list(range(120))
    assert f.query_fastx(data).records_queried == 300
