"""Saved-filter headers are read without a GPU (sbf_filter_file_info)."""
import struct

import numpy as np
import pytest


def _write(path, k=31, s=28, m=16, h=4, shards=8, version=1, magic=b"SBFB200\0", extra=0):
    hdr = magic + struct.pack("<IIIIIIQ", version, k, s, m, h, 0, shards)
    path.write_bytes(hdr + np.zeros(shards * 4 + extra, np.uint64).tobytes())


def _info(sbf, path):
    import ctypes as C

    k, s, m, h, bits = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
    st = sbf.lib().sbf_filter_file_info(str(path).encode(), C.byref(k), C.byref(s), C.byref(m),
                                        C.byref(h), C.byref(bits))
    return st, (k.value, s.value, m.value, h.value, bits.value)


def test_header_fields(sbf, tmp_path):
    p = tmp_path / "f.sbf"
    _write(p, 21, 19, 11, 4, shards=64)
    st, info = _info(sbf, p)
    assert st == 0 and info == (21, 19, 11, 4, 64 * 256)


@pytest.mark.parametrize("kw", [dict(magic=b"NOTSBF\0\0"), dict(version=9)])
def test_bad_headers(sbf, tmp_path, kw):
    p = tmp_path / "bad.sbf"
    _write(p, **kw)
    st, _ = _info(sbf, p)
    assert st == sbf.ERR_IO


def test_missing_file(sbf, tmp_path):
    st, _ = _info(sbf, tmp_path / "absent.sbf")
    assert st == sbf.ERR_IO
