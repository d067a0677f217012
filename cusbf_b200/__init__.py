"""Python host mirror of the reference cuSBF filter API over the C ABI.

``cusbf_b200.Filter`` mirrors ``cusbf::filter<Config>`` of the reference
(include/cusbf/filter.cuh of tdortman/cuSBF): the same method names, the same
argument meaning and the same error categories (raised as ``SbfError`` where
the reference returns ``cusbf::Result`` errors).  Every call goes through
libsbf_b200.so (include/sbf_b200.h); there is no CPU fallback and importing
this package fails loudly when the library has not been built.

Device buffers are passed as CUDA ``torch.Tensor`` objects (or raw integer
device pointers); host buffers as ``bytes``, ``str``, ``numpy`` arrays or
CPU tensors.  Streams are ``torch.cuda.Stream`` objects, raw ``cudaStream_t``
integers, or ``None`` for the legacy default stream.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libsbf_b200.so")

if not os.path.exists(LIBRARY_PATH):
    raise ImportError(
        f"{LIBRARY_PATH} is missing: build it with `python cusbf_b200/build.py` "
        "(the engine has no CPU fallback)")

_lib = C.CDLL(LIBRARY_PATH)

# Error categories (include/cusbf/error.hpp:67-73), offset by one.
OK = 0
ERR_CUDA = 1
ERR_IO = 2
ERR_FASTX_PARSE = 3
ERR_INVALID_ARGUMENT = 4
ERR_RESOURCE = 5
_CATEGORY = {1: "cuda", 2: "io", 3: "fastx_parse", 4: "invalid_argument", 5: "resource"}

ALPHABET_DNA = 0
ALPHABET_DNA_TRIPLET = 1
ALPHABET_PROTEIN = 2


class SbfError(RuntimeError):
    """A failed library call; ``category`` is the reference ErrorCategory name."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.category = _CATEGORY.get(status, "unknown")
        super().__init__(f"[{self.category}] {message}")


@dataclass
class Config:
    """Config<K, S, M, HashCount> (include/cusbf/config.cuh:28-118)."""

    k: int = 31
    s: int = 28
    m: int = 16
    hashes: int = 4
    alphabet: int = ALPHABET_DNA

    @property
    def minimizer_span(self) -> int:
        return self.k - self.m + 1

    @property
    def findere_span(self) -> int:
        return self.k - self.s + 1


class RecordRange(C.Structure):
    """RecordRange (include/cusbf/Fastx.hpp:24-29)."""

    _fields_ = [("sequence_offset", C.c_uint64), ("sequence_bytes", C.c_uint64)]


class InsertReport(C.Structure):
    """FastxInsertReport (include/cusbf/Fastx.hpp:151-158)."""

    _fields_ = [("records_indexed", C.c_uint64), ("indexed_bases", C.c_uint64),
                ("inserted_kmers", C.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class QueryReport(C.Structure):
    """FastxQueryReport (include/cusbf/Fastx.hpp:161-170)."""

    _fields_ = [("records_queried", C.c_uint64), ("queried_bases", C.c_uint64),
                ("queried_kmers", C.c_uint64), ("positive_kmers", C.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_vp = C.c_void_p
_u64 = C.c_uint64
_u32 = C.c_uint32


def _sig(name, res, *args):
    fn = getattr(_lib, name)
    fn.restype = res
    fn.argtypes = list(args)
    return fn


_lib_last_error = _sig("sbf_last_error_message", C.c_char_p)
_sig("sbf_last_cuda_error", C.c_int)
_sig("sbf_version", C.c_char_p)
_sig("sbf_filter_create", C.c_int, _u32, _u32, _u32, _u32, C.c_int, _u64, C.POINTER(_vp))
_sig("sbf_filter_destroy", None, _vp)
_sig("sbf_filter_clear", C.c_int, _vp, _vp)
_sig("sbf_filter_bits", _u64, _vp)
_sig("sbf_filter_num_shards", _u64, _vp)
_sig("sbf_filter_words", C.c_int, _vp, C.POINTER(_vp), C.POINTER(_u64))
_sig("sbf_filter_load_factor", C.c_int, _vp, _vp, C.POINTER(C.c_double))
_sig("sbf_filter_kmer_count", _u64, _vp, _u64)
_sig("sbf_insert_sequence_async", C.c_int, _vp, _vp, _u64, _vp, C.POINTER(_u64))
_sig("sbf_insert_sequence", C.c_int, _vp, _vp, _u64, _vp, C.POINTER(_u64))
_sig("sbf_contains_sequence_async", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp)
_sig("sbf_contains_sequence_to_device", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp)
_sig("sbf_contains_sequence", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp)
_sig("sbf_dense_packed_word_count", _u64, _u64)
_sig("sbf_pack_dense_device", C.c_int, _vp, _u64, _vp, _vp)
_sig("sbf_pack_dense_host", C.c_int, _vp, _u64, _vp)
_sig("sbf_insert_dense_packed_async", C.c_int, _vp, _vp, _u64, _u64, _vp, C.POINTER(_u64))
_sig("sbf_insert_dense_packed", C.c_int, _vp, _vp, _u64, _u64, _vp, C.POINTER(_u64))
_sig("sbf_contains_dense_packed_async", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)
_sig("sbf_contains_dense_packed_to_device", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)
_sig("sbf_contains_dense_packed", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)


def lib() -> C.CDLL:
    """The loaded libsbf_b200.so (for callers that bind extra symbols)."""
    return _lib


def version() -> str:
    return _lib.sbf_version().decode()


def _check(status: int) -> None:
    if status != OK:
        raise SbfError(status, _lib.sbf_last_error_message().decode(errors="replace"))


def _stream(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


def _dev_ptr(t) -> tuple[int, int]:
    """(device pointer, size in bytes) of a CUDA tensor or (ptr, nbytes) tuple."""
    if isinstance(t, tuple):
        return int(t[0]), int(t[1])
    if not getattr(t, "is_cuda", False):
        raise SbfError(ERR_INVALID_ARGUMENT, "expected a CUDA tensor for a device argument")
    if not t.is_contiguous():
        raise SbfError(ERR_INVALID_ARGUMENT, "device tensors must be contiguous")
    return int(t.data_ptr()), int(t.numel() * t.element_size())


def _host_bytes(seq) -> np.ndarray:
    if isinstance(seq, np.ndarray):
        return np.ascontiguousarray(seq).view(np.uint8).reshape(-1)
    if isinstance(seq, str):
        seq = seq.encode()
    if isinstance(seq, (bytes, bytearray, memoryview)):
        return np.frombuffer(seq, dtype=np.uint8)
    if hasattr(seq, "numpy"):  # CPU tensor
        return np.ascontiguousarray(seq.numpy()).view(np.uint8).reshape(-1)
    raise TypeError(f"unsupported host sequence type {type(seq)!r}")


def _np_ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Filter:
    """GPU-resident Super Bloom filter (cusbf::filter<Config>, filter.cuh:68)."""

    def __init__(self, requested_filter_bits: int, config: Config | None = None, **kw):
        self.config = config or Config(**kw)
        c = self.config
        h = _vp()
        _check(_lib.sbf_filter_create(c.k, c.s, c.m, c.hashes, c.alphabet,
                                      int(requested_filter_bits), C.byref(h)))
        self._h = h

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.sbf_filter_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- properties (filter.cuh:793-833) ------------------------------------
    def filter_bits(self) -> int:
        return _lib.sbf_filter_bits(self._h)

    def num_shards(self) -> int:
        return _lib.sbf_filter_num_shards(self._h)

    def clear(self, stream=None) -> None:
        _check(_lib.sbf_filter_clear(self._h, _stream(stream)))

    def load_factor(self, stream=None) -> float:
        out = C.c_double()
        _check(_lib.sbf_filter_load_factor(self._h, _stream(stream), C.byref(out)))
        return out.value

    def kmer_count(self, nbytes: int) -> int:
        return _lib.sbf_filter_kmer_count(self._h, nbytes)

    def words_ptr(self) -> tuple[int, int]:
        p, n = _vp(), _u64()
        _check(_lib.sbf_filter_words(self._h, C.byref(p), C.byref(n)))
        return p.value, n.value

    def words(self):
        """A uint64 CUDA tensor aliasing the shard words (no copy)."""
        import torch

        p, n = self.words_ptr()
        # Wrap the device pointer without copying via __cuda_array_interface__.
        class _View:
            __cuda_array_interface__ = {"shape": (n,), "typestr": "<u8", "data": (p, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_View(), device="cuda")

    def words_host(self) -> np.ndarray:
        """Copy of the shard words (num_shards * 4 uint64) on the host."""
        import torch

        torch.cuda.synchronize()
        return self.words().cpu().numpy().view(np.uint64).copy()

    # -- byte sequences -----------------------------------------------------
    def insert_sequence_async(self, d_seq, stream=None) -> int:
        p, n = _dev_ptr(d_seq)
        out = _u64()
        _check(_lib.sbf_insert_sequence_async(self._h, p, n, _stream(stream), C.byref(out)))
        return out.value

    def insert_sequence(self, seq, stream=None) -> int:
        b = _host_bytes(seq)
        out = _u64()
        _check(_lib.sbf_insert_sequence(self._h, _np_ptr(b), b.size, _stream(stream),
                                        C.byref(out)))
        return out.value

    def contains_sequence_async(self, d_seq, d_out, stream=None) -> None:
        p, n = _dev_ptr(d_seq)
        o, on = _dev_ptr(d_out)
        _check(_lib.sbf_contains_sequence_async(self._h, p, n, o, on, _stream(stream)))

    def contains_sequence(self, seq, d_out=None, stream=None):
        """Host sequence -> per-window bytes.  With ``d_out`` the bytes go to
        that device buffer (filter.cuh:486); otherwise a numpy array is
        returned (filter.cuh:514)."""
        b = _host_bytes(seq)
        n = self.kmer_count(b.size)
        if d_out is not None:
            o, on = _dev_ptr(d_out)
            _check(_lib.sbf_contains_sequence_to_device(self._h, _np_ptr(b), b.size, o, on,
                                                        _stream(stream)))
            return None
        out = np.zeros(max(n, 1), dtype=np.uint8)
        _check(_lib.sbf_contains_sequence(self._h, _np_ptr(b), b.size, _np_ptr(out), n,
                                          _stream(stream)))
        return out[:n]

    # -- dense packed input -------------------------------------------------
    @staticmethod
    def dense_packed_word_count(num_symbols: int) -> int:
        return _lib.sbf_dense_packed_word_count(num_symbols)

    def insert_dense_packed_async(self, d_words, num_symbols: int, stream=None) -> int:
        p, nb = _dev_ptr(d_words)
        out = _u64()
        _check(_lib.sbf_insert_dense_packed_async(self._h, p, nb // 8, num_symbols,
                                                  _stream(stream), C.byref(out)))
        return out.value

    def insert_dense_packed(self, words, num_symbols: int, stream=None) -> int:
        w = np.ascontiguousarray(words, dtype=np.uint64)
        out = _u64()
        _check(_lib.sbf_insert_dense_packed(self._h, _np_ptr(w), w.size, num_symbols,
                                            _stream(stream), C.byref(out)))
        return out.value

    def contains_dense_packed_async(self, d_words, num_symbols: int, d_out, stream=None):
        p, nb = _dev_ptr(d_words)
        o, on = _dev_ptr(d_out)
        _check(_lib.sbf_contains_dense_packed_async(self._h, p, nb // 8, num_symbols, o, on,
                                                    _stream(stream)))

    def contains_dense_packed(self, words, num_symbols: int, d_out=None, stream=None):
        w = np.ascontiguousarray(words, dtype=np.uint64)
        n = self.kmer_count(num_symbols)
        if d_out is not None:
            o, on = _dev_ptr(d_out)
            _check(_lib.sbf_contains_dense_packed_to_device(self._h, _np_ptr(w), w.size,
                                                            num_symbols, o, on, _stream(stream)))
            return None
        out = np.zeros(max(n, 1), dtype=np.uint8)
        _check(_lib.sbf_contains_dense_packed(self._h, _np_ptr(w), w.size, num_symbols,
                                              _np_ptr(out), n, _stream(stream)))
        return out[:n]


def pack_dense_sequence(seq) -> np.ndarray:
    """Host dense packing (include/cusbf/dense_packed.hpp:36-50), DNA."""
    b = _host_bytes(seq)
    n_words = _lib.sbf_dense_packed_word_count(b.size)
    out = np.zeros(max(n_words, 1), dtype=np.uint64)
    _check(_lib.sbf_pack_dense_host(_np_ptr(b), b.size, _np_ptr(out)))
    return out[:n_words]


def pack_dense_sequence_device(d_seq, num_symbols: int, d_words, stream=None) -> None:
    """Device dense packing (include/cusbf/dense_packed.hpp:58-74)."""
    p, _ = _dev_ptr(d_seq)
    w, _ = _dev_ptr(d_words)
    _check(_lib.sbf_pack_dense_device(p, num_symbols, w, _stream(stream)))


__all__ = [
    "Config", "Filter", "RecordRange", "InsertReport", "QueryReport", "SbfError",
    "pack_dense_sequence", "pack_dense_sequence_device", "lib", "version", "LIBRARY_PATH",
]
