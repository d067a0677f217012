"""FASTQ parsed on the GPU gives exactly the host parser's results: reports,
filter words, per-record views and error locations, across block boundaries
(tiny blocks), CRLF, gzip, and inputs that switch to the host parser midway
(wrapped records, blank lines, malformed tails, FASTA)."""
import gzip

import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu
K31 = dict(k=31, s=28, m=16, hashes=4)


def _fastq(rng, n, lo=20, hi=400, crlf=False, alphabet=b"ACGTACGTACGTACGTacgtN", empty_every=0):
    nl = b"\r\n" if crlf else b"\n"
    out = []
    for i in range(n):
        ln = 0 if (empty_every and i % empty_every == 0) else int(rng.integers(lo, hi))
        seq = random_dna(rng, ln, alphabet).tobytes()
        out.append(b"@r%d extra text" % i + nl + seq + nl + b"+" + nl + b"I" * ln + nl)
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


def _reads_from(rng, genome, n):
    parts = []
    for i in range(n):
        ln = int(rng.integers(20, 300))
        o = int(rng.integers(0, genome.size - ln))
        parts.append(b"@q%d\n" % i + genome[o:o + ln].tobytes() + b"\n+\n" + b"#" * ln + b"\n")
    return b"".join(parts)


@pytest.mark.parametrize("block", [4096, 5000, 65536, 0])
@pytest.mark.parametrize("crlf", [False, True])
def test_query_matches_host_parser(sbf, cuda, monkeypatch, block, crlf):
    rng = np.random.default_rng(block + crlf)
    genome = random_dna(rng, 200_000)
    data = _reads_from(rng, genome, 300) + _fastq(rng, 300, crlf=False)
    if crlf:
        data = data.replace(b"\n", b"\r\n")
    dev = _run(sbf, monkeypatch, "device", block, data, genome)
    host = _run(sbf, monkeypatch, "host", 0, data, genome)
    _same(dev, host)
    assert dev[0]["positive_kmers"] > 0


@pytest.mark.parametrize("block", [4096, 0])
def test_insert_matches_host_parser(sbf, cuda, monkeypatch, tmp_path, block):
    rng = np.random.default_rng(7)
    data = _fastq(rng, 500, empty_every=37)
    p = tmp_path / "in.fq.gz"
    p.write_bytes(gzip.compress(data))
    genome = random_dna(rng, 1000)
    dev = _run(sbf, monkeypatch, "device", block, str(p), genome, query=False, as_file=True)
    host = _run(sbf, monkeypatch, "host", 0, str(p), genome, query=False, as_file=True)
    _same(dev, host)
    assert dev[0]["records_indexed"] == 500


@pytest.mark.parametrize("kind", ["wrapped", "blank-lines", "fasta", "no-final-newline"])
def test_switches_to_host_parser(sbf, cuda, monkeypatch, kind):
    rng = np.random.default_rng(11)
    genome = random_dna(rng, 100_000)
    head = _reads_from(rng, genome, 200)
    if kind == "wrapped":
        tail = b"@w\nACGTACGTACGTACGTACGTACGTACGTAC\nGTACGTACGTACGTACGTACGT\n+\n" + b"I" * 30 + b"\n" + b"I" * 22 + b"\n"
    elif kind == "blank-lines":
        tail = b"\n\n" + _reads_from(rng, genome, 50)
    elif kind == "fasta":
        head, tail = b"", b">s\n" + genome[:5000].tobytes() + b"\n>t\n" + genome[9000:9400].tobytes() + b"\n"
    else:
        tail = b"@last\n" + genome[:100].tobytes() + b"\n+\n" + b"I" * 100
    data = head + tail + _reads_from(rng, genome, 20) if kind in ("wrapped", "blank-lines") else head + tail
    dev = _run(sbf, monkeypatch, "device", 4096, data, genome)
    host = _run(sbf, monkeypatch, "host", 0, data, genome)
    _same(dev, host)


def test_error_locations_match(sbf, cuda, monkeypatch):
    rng = np.random.default_rng(13)
    genome = random_dna(rng, 50_000)
    data = _reads_from(rng, genome, 400) + b"@broken\nACGTACGT\n+\nIIIIIII\n"
    errs = []
    for parser, block in (("device", 4096), ("host", 0)):
        monkeypatch.setenv("SBF_FASTX_PARSER", parser)
        monkeypatch.setenv("SBF_FASTQ_BLOCK_BYTES", str(block or 1 << 20))
        f = sbf.Filter(1 << 20, **K31)
        with pytest.raises(sbf.SbfError) as ei:
            f.query_fastx(data, source_name="x.fq")
        errs.append((str(ei.value), ei.value.location))
    assert errs[0] == errs[1]
    assert errs[0][1][1] == 4 * 400 + 4


def test_abort_from_consumer(sbf, cuda, monkeypatch):
    monkeypatch.setenv("SBF_FASTQ_BLOCK_BYTES", "4096")
    rng = np.random.default_rng(17)
    genome = random_dna(rng, 50_000)
    data = _reads_from(rng, genome, 300)
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
