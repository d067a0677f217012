"""FASTA/FASTQ parsing on the host (CPU).  Cases restate the reference's
tests/test_fastx.cu inputs; expected records follow include/cusbf/Fastx.hpp."""
import gzip

import pytest


def test_wrapped_fasta(sbf):
    # test_fastx.cu:23-41
    assert sbf.fastx_scan(">wrapped\nACGT\nACGT\nACGT\n") == [("wrapped", b"ACGTACGTACGT")]


def test_fastq_crlf_wrapped(sbf):
    # test_fastx.cu:43-64
    recs = sbf.fastx_scan("@wrapped\r\nACGTAC\r\nGTACGT\r\n+\r\nIIIIII\r\nIIIIII\r\n")
    assert recs == [("wrapped", b"ACGTACGTACGT")]


def test_multi_record_and_blank_lines(sbf):
    recs = sbf.fastx_scan("\n\n>first\nACGT\n\nACGT\n>second\nTGCA\nTGCA")
    assert recs == [("first", b"ACGTACGT"), ("second", b"TGCATGCA")]


def test_quality_line_starting_with_at(sbf):
    recs = sbf.fastx_scan("@r\nACGT\n+\n@@@@\n@s\nTT\n+comment\nII\n")
    assert recs == [("r", b"ACGT"), ("s", b"TT")]


def test_malformed_quality_location(sbf):
    # test_fastx.cu:708-727: line 4, column 8
    with pytest.raises(sbf.SbfError) as e:
        sbf.fastx_scan("@broken\nACGTACGT\n+\nIIIIIII\n", "broken.fq")
    assert e.value.category == "fastx_parse"
    assert e.value.location == ("broken.fq", 4, 8)


def test_quality_too_long(sbf):
    with pytest.raises(sbf.SbfError) as e:
        sbf.fastx_scan("@r\nACGT\n+\nIIIIII\n", "x")
    assert e.value.category == "fastx_parse" and "exceeds" in e.value.message
    assert e.value.location == ("x", 4, 5)


def test_unterminated_and_mixed(sbf):
    with pytest.raises(sbf.SbfError) as e:
        sbf.fastx_scan("@r\nACGT\n")
    assert "missing '+'" in e.value.message
    # A '>' header after FASTQ records is rejected; inside FASTA records an
    # '@' line is sequence, as in the reference reader.
    with pytest.raises(sbf.SbfError) as e:
        sbf.fastx_scan("@a\nAC\n+\nII\n>b\nACGT\n")
    assert "mixed FASTA and FASTQ" in e.value.message
    assert sbf.fastx_scan(">a\nACGT\n@b\n") == [("a", b"ACGT@b")]
    with pytest.raises(sbf.SbfError) as e:
        sbf.fastx_scan("xACGT\n")
    assert "expected FASTA or FASTQ header" in e.value.message


def test_gzip_and_plain_files(sbf, tmp_path):
    text = b">a\nACGTACGT\n>b\nTTTT\n"
    plain = tmp_path / "x.fa"
    plain.write_bytes(text)
    gz = tmp_path / "x.fa.gz"
    gz.write_bytes(gzip.compress(text))
    assert sbf.fastx_scan_file(plain) == sbf.fastx_scan_file(gz) == [("a", b"ACGTACGT"),
                                                                     ("b", b"TTTT")]
    with pytest.raises(sbf.SbfError) as e:
        sbf.fastx_scan_file(tmp_path / "missing.fa")
    assert e.value.category == "io"


def test_large_stream_crosses_buffers(sbf):
    import io

    recs = [(f"r{i}", (b"ACGT" * (i % 50 + 1))) for i in range(20000)]
    text = b"".join(b">" + h.encode() + b"\n" + s + b"\n" for h, s in recs)
    assert sbf.fastx_scan(io.BytesIO(text)) == recs


def test_large_plain_file_matches_gzip_and_stream(sbf, tmp_path):
    """An uncompressed file is read with pread() (here in the host parser's
    4 MiB chunks), a gzip file through zlib: the records of a 15 MB file equal
    those of the same bytes read both ways and through a stream."""
    import gzip

    import numpy as np

    rng = np.random.default_rng(5)
    parts = []
    for i in range(3000):
        seq = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(rng.integers(1000, 9000)))]
        lines = [seq[j:j + 70].tobytes() for j in range(0, seq.size, 70)]
        parts.append(b">r%d\n" % i + b"\n".join(lines) + b"\n")
    data = b"".join(parts)
    assert len(data) > 3 * (4 << 20)
    plain = tmp_path / "big.fa"
    plain.write_bytes(data)
    gz = tmp_path / "big.fa.gz"
    gz.write_bytes(gzip.compress(data, compresslevel=1))
    a = sbf.fastx_scan_file(plain)
    b = sbf.fastx_scan_file(gz)
    c = sbf.fastx_scan(data)
    assert len(a) == 3000 and a == b == c
