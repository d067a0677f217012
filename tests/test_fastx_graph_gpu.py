"""FASTQ and FASTA blocks replayed as one CUDA graph each (upload, newline
scan, record parse, ragged insert or query, one download) give exactly the
stream-launched device path's and the host parser's results: reports and
filter words, across block boundaries, records longer than a block,
irregular input that switches to the host parser, and line tables that
overflow and are grown."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu
K31 = dict(k=31, s=28, m=16, hashes=4)


def _fastq(rng, n, lo=20, hi=400):
    out = []
    for i in range(n):
        ln = int(rng.integers(lo, hi))
        seq = random_dna(rng, ln, b"ACGTACGTACGTACGTacgtN").tobytes()
        out.append(b"@r%d x\n" % i + seq + b"\n+\n" + b"I" * ln + b"\n")
    return b"".join(out)


def _fasta(rng, n, lo=50, hi=3000, width=60):
    out = []
    for i in range(n):
        seq = random_dna(rng, int(rng.integers(lo, hi)), b"ACGTACGTACGTacgtN").tobytes()
        lines = [seq[j:j + width] for j in range(0, len(seq), width)] or [b""]
        out.append(b">s%d\n" % i + b"\n".join(lines) + b"\n")
    return b"".join(out)


def _run(sbf, monkeypatch, mode, block, data, genome, query):
    monkeypatch.setenv("SBF_FASTX_PARSER", "host" if mode == "host" else "device")
    monkeypatch.setenv("SBF_FASTX_GRAPH", "1" if mode == "graph" else "0")
    if block:
        monkeypatch.setenv("SBF_FASTQ_BLOCK_BYTES", str(block))
    else:
        monkeypatch.delenv("SBF_FASTQ_BLOCK_BYTES", raising=False)
    f = sbf.Filter(1 << 22, **K31)
    f.insert_sequence(genome)
    rep = f.query_fastx(data) if query else f.insert_fastx(data)
    return rep.as_dict(), f.words_host()


@pytest.mark.parametrize("fmt", ["fastq", "fasta"])
@pytest.mark.parametrize("query", [True, False])
@pytest.mark.parametrize("block", [4096, 70000, 0])
def test_graph_equals_stream_and_host(sbf, cuda, monkeypatch, fmt, query, block):
    rng = np.random.default_rng((1 if fmt == "fastq" else 2) * 1000 + 10 * query + block % 7)
    genome = random_dna(rng, 200_000)
    data = _fastq(rng, 3000) if fmt == "fastq" else _fasta(rng, 400)
    runs = {m: _run(sbf, monkeypatch, m, block, data, genome, query)
            for m in ("graph", "stream", "host")}
    for m in ("stream", "host"):
        assert runs["graph"][0] == runs[m][0], m
        np.testing.assert_array_equal(runs["graph"][1], runs[m][1])
    assert runs["graph"][0]["records_queried" if query else "records_indexed"] > 0


@pytest.mark.parametrize("query", [True, False])
def test_graph_falls_back_on_irregular_input(sbf, cuda, monkeypatch, query):
    rng = np.random.default_rng(7)
    genome = random_dna(rng, 100_000)
    # Regular records, then a wrapped FASTQ record and more records.
    head = _fastq(rng, 500)
    tail = b"@wrapped\nACGTACGTAC\nGTACGT\n+\nIIIIIIIIII\nIIIIII\n" + _fastq(rng, 200)
    data = head + tail
    g = _run(sbf, monkeypatch, "graph", 8192, data, genome, query)
    h = _run(sbf, monkeypatch, "host", 8192, data, genome, query)
    assert g[0] == h[0]
    np.testing.assert_array_equal(g[1], h[1])


def test_graph_grows_the_line_table(sbf, cuda, monkeypatch):
    """A block of very short lines has more newlines than the first line-table
    estimate (len / 32): the block is run again after the table grows."""
    rng = np.random.default_rng(11)
    genome = random_dna(rng, 50_000)
    recs = []
    for i in range(4000):
        seq = random_dna(rng, 40, b"ACGT").tobytes()
        recs.append(b">" + b"\n".join(seq[j:j + 2] for j in range(0, 40, 2)) + b"\n")
    data = b"".join(recs)
    g = _run(sbf, monkeypatch, "graph", 0, data, genome, True)
    h = _run(sbf, monkeypatch, "host", 0, data, genome, True)
    assert g[0] == h[0]
    np.testing.assert_array_equal(g[1], h[1])


@pytest.mark.parametrize("query", [True, False])
def test_large_plain_file_device_equals_host_parser(sbf, cuda, monkeypatch, tmp_path, query):
    """A 40 MB uncompressed FASTQ file: the device parser reads its blocks
    with parallel pread() slices (files above 8 MiB), the host parser in 4 MiB
    chunks; reports and filter words must agree."""
    rng = np.random.default_rng(99)
    genome = random_dna(rng, 500_000)
    path = tmp_path / "reads.fq"
    path.write_bytes(_fastq(rng, 150_000, 100, 400))
    assert path.stat().st_size > 5 * (8 << 20)
    out = {}
    for mode in ("graph", "host"):
        monkeypatch.setenv("SBF_FASTX_PARSER", "host" if mode == "host" else "device")
        monkeypatch.setenv("SBF_FASTQ_BLOCK_BYTES", str(16 << 20))
        f = sbf.Filter(1 << 22, **K31)
        f.insert_sequence(genome)
        rep = f.query_fastx_file(str(path)) if query else f.insert_fastx_file(str(path))
        out[mode] = (rep.as_dict(), f.words_host())
    assert out["graph"][0] == out["host"][0]
    np.testing.assert_array_equal(out["graph"][1], out["host"][1])
