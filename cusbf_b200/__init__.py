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
import threading
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
ERR_ABORTED = 6
_CATEGORY = {1: "cuda", 2: "io", 3: "fastx_parse", 4: "invalid_argument", 5: "resource",
             6: "aborted"}

ALPHABET_DNA = 0
ALPHABET_DNA_TRIPLET = 1
ALPHABET_PROTEIN = 2


class SbfError(RuntimeError):
    """A failed library call; ``category`` is the reference ErrorCategory name
    and ``location`` the (file, line, column) of a FASTX parse error."""

    def __init__(self, status: int, message: str, location=None):
        self.status = status
        self.category = _CATEGORY.get(status, "unknown")
        self.message = message
        self.location = location
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


class RaggedTuning(C.Structure):
    """sbf_ragged_tuning: host-pipeline knobs of ragged batches (0 = default)."""

    _fields_ = [("chunk_bytes", C.c_uint64), ("stages", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("use_graph", C.c_uint32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerConfig(C.Structure):
    """sbf_server_config (0 = default)."""

    _fields_ = [("staging_bytes", C.c_uint64), ("max_batch_bytes", C.c_uint64),
                ("pinned_bytes", C.c_uint64), ("max_inflight", C.c_uint32),
                ("max_batch_requests", C.c_uint32), ("use_graph", C.c_uint32)]


class ServerRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("latency_s", C.c_double), ("windows", C.c_uint64),
                ("arrival_s", C.c_double), ("done_s", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("batches", C.c_uint64),
                ("query_windows", C.c_uint64), ("insert_windows", C.c_uint64),
                ("wall_s", C.c_double), ("p50_s", C.c_double), ("p99_s", C.c_double),
                ("p999_s", C.c_double), ("max_s", C.c_double), ("mean_s", C.c_double),
                ("mean_batch_requests", C.c_double), ("worker_busy_s", C.c_double),
                ("admission_wait_s", C.c_double), ("slot_wait_s", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class NormalizedRecord(C.Structure):
    """NormalizedRecord (include/cusbf/normalized_record_batch.hpp:20-29)."""

    _fields_ = [("record_index", C.c_uint64), ("input_offset", C.c_uint64),
                ("size", C.c_uint64), ("valid_kmers", C.c_uint64)]


class QueryLayoutRecord(C.Structure):
    """QueryLayoutRecord (include/cusbf/detail/query_layout.cuh:13-20)."""

    _fields_ = [("record_index", C.c_uint64), ("input_offset", C.c_uint64),
                ("size", C.c_uint64), ("valid_kmers", C.c_uint64),
                ("hit_offset", C.c_uint64), ("hit_count", C.c_uint64)]


class RecordView(C.Structure):
    """RecordQueryView (include/cusbf/Fastx.hpp:135-148), valid during a callback."""

    _fields_ = [("record_index", C.c_uint64), ("sequence", C.c_void_p),
                ("sequence_bytes", C.c_uint64), ("queried_bases", C.c_uint64),
                ("queried_kmers", C.c_uint64), ("positive_kmers", C.c_uint64),
                ("hits", C.c_void_p), ("n_hits", C.c_uint64)]


RECORD_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(RecordView))


class FastxRecordView(C.Structure):
    """FastxRecordView (include/cusbf/Fastx.hpp:173-188), valid during a callback."""

    _fields_ = [("record_index", C.c_uint64), ("header", C.c_void_p),
                ("header_bytes", C.c_uint64), ("sequence", C.c_void_p),
                ("sequence_bytes", C.c_uint64), ("queried_bases", C.c_uint64),
                ("queried_kmers", C.c_uint64), ("positive_kmers", C.c_uint64),
                ("hits", C.c_void_p), ("n_hits", C.c_uint64)]


FASTX_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(FastxRecordView))
SCAN_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
                      C.c_uint64)
READ_FN = C.CFUNCTYPE(C.c_int64, C.c_void_p, C.c_void_p, C.c_uint64)

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
_sig("sbf_last_error_location", C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_uint32),
     C.POINTER(C.c_uint32))
_sig("sbf_version", C.c_char_p)
_sig("sbf_filter_create", C.c_int, _u32, _u32, _u32, _u32, C.c_int, _u64, C.POINTER(_vp))
_sig("sbf_filter_destroy", None, _vp)
_sig("sbf_filter_clear", C.c_int, _vp, _vp)
_sig("sbf_filter_bits", _u64, _vp)
_sig("sbf_filter_num_shards", _u64, _vp)
_sig("sbf_filter_kernel_path", C.c_int, _vp)
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
_sig("sbf_dense_packed_word_count_for", _u64, C.c_int, _u64)
_sig("sbf_contains_dense_packed_bits_async", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)
_sig("sbf_contains_dense_packed_bits", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)
_sig("sbf_pack_dense_device_for", C.c_int, C.c_int, _vp, _u64, _vp, _vp)
_sig("sbf_pack_dense_host_for", C.c_int, C.c_int, _vp, _u64, _vp)
_sig("sbf_insert_dense_packed_async", C.c_int, _vp, _vp, _u64, _u64, _vp, C.POINTER(_u64))
_sig("sbf_insert_dense_packed", C.c_int, _vp, _vp, _u64, _u64, _vp, C.POINTER(_u64))
_sig("sbf_contains_dense_packed_async", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)
_sig("sbf_contains_dense_packed_to_device", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)
_sig("sbf_contains_dense_packed", C.c_int, _vp, _vp, _u64, _u64, _vp, _u64, _vp)
_sig("sbf_validate_record_batch", C.c_int, _u64, _vp, _u64)
_sig("sbf_normalized_batch_bytes", _u64, _vp, _u64)
_sig("sbf_normalize_record_batch", C.c_int, _u32, _vp, _u64, _vp, _u64, _vp, _u64,
     C.POINTER(_u64), _vp)
_sig("sbf_query_layout", C.c_int, _u32, _vp, _u64, _vp, C.POINTER(_u64))
_sig("sbf_validate_record_batch_for", C.c_int, C.c_int, _u64, _vp, _u64)
_sig("sbf_normalized_batch_bytes_for", _u64, C.c_int, _vp, _u64)
_sig("sbf_normalize_record_batch_for", C.c_int, C.c_int, _u32, _vp, _u64, _vp, _u64, _vp, _u64,
     C.POINTER(_u64), _vp)
_sig("sbf_query_layout_for", C.c_int, C.c_int, _u32, _vp, _u64, _vp, C.POINTER(_u64))
_sig("sbf_insert_record_batch", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, C.POINTER(InsertReport))
_sig("sbf_insert_record_batch_async", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, C.POINTER(_u64))
_sig("sbf_query_record_batch", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, C.POINTER(QueryReport),
     RECORD_CB, _vp)
_sig("sbf_contains_record_batch_async", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _vp)
_sig("sbf_ragged_insert_async", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, _vp)
_sig("sbf_ragged_contains_async", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _vp, _vp)
_sig("sbf_ragged_contains_counts_async", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _vp, _vp,
     _vp, _vp)
_sig("sbf_ragged_insert", C.c_int, _vp, _vp, _u64, _vp, _u64, C.POINTER(RaggedTuning), _vp,
     C.POINTER(InsertReport))
_sig("sbf_ragged_query", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, _u64, C.POINTER(RaggedTuning),
     _vp, C.POINTER(QueryReport))
_sig("sbf_ragged_query_bits", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, _u64, C.POINTER(RaggedTuning),
     _vp, C.POINTER(QueryReport))
_sig("sbf_ragged_autotune", C.c_int, _vp, C.c_int, _vp, _u64, _vp, _u64, _u64, _vp,
     C.POINTER(RaggedTuning))
_sig("sbf_ragged_tuning_lookup", C.c_int, _vp, C.c_int, _u64, _u64, C.POINTER(RaggedTuning))
_sig("sbf_server_create", C.c_int, _vp, C.POINTER(ServerConfig), C.POINTER(_vp))
_sig("sbf_server_destroy", None, _vp)
_sig("sbf_server_now", C.c_double)
_sig("sbf_server_submit", C.c_int, _vp, C.c_int, _vp, _vp, _u64, _vp, _u64, C.c_double,
     C.POINTER(_u64))
_sig("sbf_server_wait", C.c_int, _vp, _u64, C.c_double, C.POINTER(ServerRequestInfo))
_sig("sbf_server_drain", C.c_int, _vp)
_sig("sbf_server_get_stats", C.c_int, _vp, C.c_int, C.POINTER(ServerStats))
_sig("sbf_contains_sequence_bits_async", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp)
_sig("sbf_emit_runs_async", C.c_int, _vp, _vp, _u64, _vp, _vp, _u64, _vp, _vp)
_sig("sbf_apply_runs_async", C.c_int, _vp, _vp, _vp, _u64, _u64, _u64, _vp)
_sig("sbf_filter_synchronize", C.c_int, _vp, _vp)
_sig("sbf_contains_sequence_bits", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp)
_sig("sbf_expand_result_bits", C.c_int, _vp, _u64, _vp, _u32)
_sig("sbf_host_expand_threads", C.c_int)
_sig("sbf_filter_save", C.c_int, _vp, C.c_char_p, _vp)
_sig("sbf_filter_file_info", C.c_int, C.c_char_p, C.POINTER(_u32), C.POINTER(_u32),
     C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_u64))
_sig("sbf_filter_load", C.c_int, _vp, C.c_char_p, _vp)
_sig("sbf_record_batch_counts_noalloc", C.c_int, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _vp,
     _vp, _vp)
_sig("sbf_fastx_scan", C.c_int, READ_FN, _vp, C.c_char_p, SCAN_CB, _vp, C.POINTER(_u64))
_sig("sbf_fastx_scan_file", C.c_int, C.c_char_p, SCAN_CB, _vp, C.POINTER(_u64))
_sig("sbf_insert_fastx", C.c_int, _vp, READ_FN, _vp, C.c_char_p, C.c_double, _vp,
     C.POINTER(InsertReport))
_sig("sbf_insert_fastx_file", C.c_int, _vp, C.c_char_p, C.c_double, _vp, C.POINTER(InsertReport))
_sig("sbf_query_fastx", C.c_int, _vp, READ_FN, _vp, C.c_char_p, C.c_double, _vp,
     C.POINTER(QueryReport), FASTX_CB, _vp)
_sig("sbf_query_fastx_file", C.c_int, _vp, C.c_char_p, C.c_double, _vp, C.POINTER(QueryReport),
     FASTX_CB, _vp)


def lib() -> C.CDLL:
    """The loaded libsbf_b200.so (for callers that bind extra symbols)."""
    return _lib


def version() -> str:
    return _lib.sbf_version().decode()


def _check(status: int) -> None:
    if status != OK:
        loc = None
        if status == ERR_FASTX_PARSE:
            f, ln, col = C.c_char_p(), _u32(), _u32()
            _lib.sbf_last_error_location(C.byref(f), C.byref(ln), C.byref(col))
            loc = ((f.value or b"").decode(errors="replace"), ln.value, col.value)
        raise SbfError(status, _lib.sbf_last_error_message().decode(errors="replace"), loc)


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


def _ranges(ranges) -> np.ndarray:
    """(n, 2) uint64 array of (sequence_offset, sequence_bytes) pairs."""
    r = np.ascontiguousarray(np.asarray(ranges, dtype=np.uint64).reshape(-1, 2))
    return r


def records_from_ranges(seq, ranges):
    """RecordBatchView-style helper: the records a (sequence, ranges) pair names."""
    b = _host_bytes(seq)
    return [b[int(o):int(o) + int(n)] for o, n in _ranges(ranges)]


def validate_record_batch(nbytes: int, ranges, alphabet: int = ALPHABET_DNA) -> None:
    r = _ranges(ranges)
    _check(_lib.sbf_validate_record_batch_for(alphabet, nbytes, _np_ptr(r), r.shape[0]))


def normalized_batch_bytes(ranges, alphabet: int = ALPHABET_DNA) -> int:
    r = _ranges(ranges)
    return _lib.sbf_normalized_batch_bytes_for(alphabet, _np_ptr(r), r.shape[0])


def normalize_record_batch(k: int, seq, ranges, alphabet: int = ALPHABET_DNA):
    """normalize_record_batch (normalized_record_batch.hpp:289-316): the
    separator-joined sequence and one NormalizedRecord per record."""
    b = _host_bytes(seq)
    r = _ranges(ranges)
    n = r.shape[0]
    total = _u64()
    recs = (NormalizedRecord * max(n, 1))()
    _check(_lib.sbf_normalize_record_batch_for(alphabet, k, _np_ptr(b), b.size, _np_ptr(r), n,
                                               None, 0, C.byref(total), None))
    out = np.zeros(max(total.value, 1), dtype=np.uint8)
    _check(_lib.sbf_normalize_record_batch_for(alphabet, k, _np_ptr(b), b.size, _np_ptr(r), n,
                                               _np_ptr(out), out.size, C.byref(total), recs))
    return out[:total.value], list(recs)[:n]


def query_layout(k: int, records, alphabet: int = ALPHABET_DNA):
    """QueryLayout::build (query_layout.cuh:42-72): (layout records, total hits)."""
    n = len(records)
    arr = (NormalizedRecord * max(n, 1))(*records)
    out = (QueryLayoutRecord * max(n, 1))()
    total = _u64()
    _check(_lib.sbf_query_layout_for(alphabet, k, arr, n, out, C.byref(total)))
    return list(out)[:n], total.value


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

    KERNELS_COMPILED, KERNELS_RUNTIME_COMPILED, KERNELS_GENERIC = 0, 1, 2

    def kernel_path(self) -> int:
        """0: tile kernels compiled into the library; 1: the same kernels
        compiled at run time for this configuration; 2: the
        runtime-parameterised kernels.  Results are identical."""
        return _lib.sbf_filter_kernel_path(self._h)

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
    def dense_packed_word_count(num_symbols: int, alphabet: int = ALPHABET_DNA) -> int:
        """Words of `num_symbols` dense symbols (64 / symbolBits per word)."""
        return _lib.sbf_dense_packed_word_count_for(alphabet, num_symbols)

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

    def contains_dense_packed_bits_async(self, d_words, num_symbols: int, d_bits,
                                         stream=None) -> None:
        """Dense input, one result bit per window (bit i % 32 of word i / 32)."""
        p, nb = _dev_ptr(d_words)
        o, on = _dev_ptr(d_bits)
        _check(_lib.sbf_contains_dense_packed_bits_async(self._h, p, nb // 8, num_symbols, o,
                                                         on // 4, _stream(stream)))

    def contains_dense_packed_bits(self, words, num_symbols: int, out=None, stream=None):
        """Host dense words -> uint32 result words (one bit per window)."""
        w = np.ascontiguousarray(words, dtype=np.uint64)
        n = max(num_symbols - self.config.k + 1, 0)
        nw = (n + 31) // 32
        if out is None:
            out = np.zeros(max(nw, 1), np.uint32)
        o = out.numpy() if hasattr(out, "numpy") else out
        _check(_lib.sbf_contains_dense_packed_bits(self._h, _np_ptr(w), w.size, num_symbols,
                                                   _np_ptr(o), o.nbytes // 4, _stream(stream)))
        return o[:nw]

    def contains_dense_packed(self, words, num_symbols: int, d_out=None, stream=None):
        w = np.ascontiguousarray(words, dtype=np.uint64)
        n = max(num_symbols - self.config.k + 1, 0)
        if d_out is not None:
            o, on = _dev_ptr(d_out)
            _check(_lib.sbf_contains_dense_packed_to_device(self._h, _np_ptr(w), w.size,
                                                            num_symbols, o, on, _stream(stream)))
            return None
        out = np.zeros(max(n, 1), dtype=np.uint8)
        _check(_lib.sbf_contains_dense_packed(self._h, _np_ptr(w), w.size, num_symbols,
                                              _np_ptr(out), n, _stream(stream)))
        return out[:n]


def _record_methods():
    def insert_record_batch(self, seq, ranges, stream=None) -> InsertReport:
        """insert_record_batch (filter.cuh:338-364): host records."""
        b = _host_bytes(seq)
        r = _ranges(ranges)
        rep = InsertReport()
        _check(_lib.sbf_insert_record_batch(self._h, _np_ptr(b), b.size, _np_ptr(r), r.shape[0],
                                            _stream(stream), C.byref(rep)))
        return rep

    def insert_record_batch_async(self, d_seq, ranges, stream=None) -> int:
        """insert_record_batch_async (filter.cuh:385-400): separators in place."""
        p, n = _dev_ptr(d_seq)
        r = _ranges(ranges)
        out = _u64()
        _check(_lib.sbf_insert_record_batch_async(self._h, p, n, _np_ptr(r), r.shape[0],
                                                  _stream(stream), C.byref(out)))
        return out.value

    def query_record_batch(self, seq, ranges, consume=None, stream=None) -> QueryReport:
        """query_record_batch (filter.cuh:549-582).  `consume(view)` receives a
        dict per record: record_index, sequence (bytes), queried_bases,
        queried_kmers, positive_kmers, hits (numpy copy)."""
        b = _host_bytes(seq)
        r = _ranges(ranges)
        rep = QueryReport()
        cb = RECORD_CB()
        box = []
        if consume is not None:
            def _cb(_user, view_p):
                v = view_p.contents
                hits = (np.ctypeslib.as_array(C.cast(v.hits, C.POINTER(C.c_uint8)), (v.n_hits,)).copy()
                        if v.n_hits else np.zeros(0, np.uint8))
                seqb = C.string_at(v.sequence, v.sequence_bytes) if v.sequence_bytes else b""
                try:
                    consume({"record_index": v.record_index, "sequence": seqb,
                             "queried_bases": v.queried_bases, "queried_kmers": v.queried_kmers,
                             "positive_kmers": v.positive_kmers, "hits": hits})
                    return 0
                except BaseException as e:  # noqa: BLE001 - re-raised after the call
                    box.append(e)
                    return 1
            cb = RECORD_CB(_cb)
        st = _lib.sbf_query_record_batch(self._h, _np_ptr(b), b.size, _np_ptr(r), r.shape[0],
                                         _stream(stream), C.byref(rep), cb, None)
        if box:
            raise box[0]
        _check(st)
        return rep

    def contains_record_batch_async(self, d_seq, ranges, d_out, stream=None) -> None:
        """contains_record_batch_async (filter.cuh:603-622)."""
        p, n = _dev_ptr(d_seq)
        o, on = _dev_ptr(d_out)
        r = _ranges(ranges)
        _check(_lib.sbf_contains_record_batch_async(self._h, p, n, _np_ptr(r), r.shape[0], o, on,
                                                    _stream(stream)))

    def record_batch_counts_noalloc(self, d_seq, ranges, d_hits=None, stream=None):
        """Per-record (valid, positive) k-mer counts of a device record batch,
        allocating nothing (sbf_record_batch_counts_noalloc; at most 262144
        records; calls on one device must not overlap)."""
        p, n = _dev_ptr(d_seq)
        h, hn = _dev_ptr(d_hits) if d_hits is not None else (None, 0)
        r = _ranges(ranges)
        valid = np.zeros(r.shape[0], np.uint64)
        pos = np.zeros(r.shape[0], np.uint64)
        _check(_lib.sbf_record_batch_counts_noalloc(self._h, p, n, _np_ptr(r), r.shape[0], h, hn,
                                                    _stream(stream), _np_ptr(valid),
                                                    _np_ptr(pos)))
        return valid, pos

    for f in (insert_record_batch, insert_record_batch_async, query_record_batch,
              contains_record_batch_async, record_batch_counts_noalloc):
        setattr(Filter, f.__name__, f)


_record_methods()


def _tuning(t):
    if t is None:
        return None
    if isinstance(t, RaggedTuning):
        return C.byref(t)
    return C.byref(RaggedTuning(**t))


def _persist_methods():
    """Filter persistence (sbf_filter_save / sbf_filter_load)."""

    def save(self, path, stream=None) -> None:
        _check(_lib.sbf_filter_save(self._h, os.fsencode(path), _stream(stream)))

    def load_words(self, path, stream=None) -> None:
        """Replaces this filter's words with a saved filter of the same
        configuration and size."""
        _check(_lib.sbf_filter_load(self._h, os.fsencode(path), _stream(stream)))

    def load(cls, path, stream=None) -> "Filter":
        """A new filter holding a saved filter."""
        k, s, m, h, bits = _u32(), _u32(), _u32(), _u32(), _u64()
        _check(_lib.sbf_filter_file_info(os.fsencode(path), C.byref(k), C.byref(s), C.byref(m),
                                         C.byref(h), C.byref(bits)))
        f = cls(bits.value, k=k.value, s=s.value, m=m.value, hashes=h.value)
        f.load_words(path, stream)
        return f

    def contains_sequence_bits_async(self, d_seq, d_bits, stream=None) -> None:
        """Bit-packed query of device bytes into a device int32/uint32 tensor:
        bit i % 32 of word i // 32 is window i's hit."""
        p, n = _dev_ptr(d_seq)
        o, on = _dev_ptr(d_bits)
        _check(_lib.sbf_contains_sequence_bits_async(self._h, p, n, o, on // 4, _stream(stream)))

    def contains_sequence_bits(self, seq, out=None, stream=None) -> np.ndarray:
        """Bit-packed query of host bytes; returns uint32 words."""
        b = _host_bytes(seq)
        n_words = (self.kmer_count(b.size) + 31) // 32
        o = np.zeros(max(n_words, 1), np.uint32) if out is None else out
        _check(_lib.sbf_contains_sequence_bits(self._h, _np_ptr(b), b.size, _np_ptr(o), o.size,
                                               _stream(stream)))
        return o[:n_words]

    Filter.contains_sequence_bits_async = contains_sequence_bits_async
    Filter.contains_sequence_bits = contains_sequence_bits
    Filter.save = save
    Filter.load_words = load_words
    Filter.load = classmethod(load)


_persist_methods()


def _sharded_methods():
    """Device steps of the sharded multi-rank insert (cusbf_b200.sharded)."""

    def emit_runs(self, d_seq, stream=None):
        """Run records of the windows of device bytes `d_seq`: (shards int32
        CUDA tensor (R,), masks int64 CUDA tensor (R, 4), valid windows)."""
        import torch

        p, n = _dev_ptr(d_seq)
        dev = d_seq.device
        cap = max(self.kmer_count(n) // 4 + 4096, 1)
        count = torch.zeros(2, dtype=torch.int64, device=dev)
        while True:
            shards = torch.empty(cap, dtype=torch.int32, device=dev)
            masks = torch.empty((cap, 4), dtype=torch.int64, device=dev)
            # The count buffer is written on torch's current stream and read
            # back after the launch on `stream`, which may be another one.
            torch.cuda.current_stream(dev).synchronize()
            _check(_lib.sbf_emit_runs_async(self._h, p, n, shards.data_ptr(), masks.data_ptr(),
                                            cap, count.data_ptr(), _stream(stream)))
            self.synchronize(stream)
            got = count.tolist()
            if got[0] <= cap:
                return shards[:got[0]], masks[:got[0]], int(got[1])
            cap = got[0]

    def apply_runs(self, d_shards, d_masks, shard_lo: int, shard_hi: int, stream=None) -> None:
        """ORs device run records (int32 shards (R,), int64 masks (R, 4)) whose
        shards lie in [shard_lo, shard_hi) into this filter."""
        s, _ = _dev_ptr(d_shards)
        m, mn = _dev_ptr(d_masks)
        _check(_lib.sbf_apply_runs_async(self._h, s, m, mn // 32, shard_lo, shard_hi,
                                         _stream(stream)))

    def synchronize(self, stream=None) -> None:
        """Waits for `stream`; raises on a device-side error of this filter."""
        _check(_lib.sbf_filter_synchronize(self._h, _stream(stream)))

    Filter.emit_runs = emit_runs
    Filter.apply_runs = apply_runs
    Filter.synchronize = synchronize


_sharded_methods()


def _ragged_methods():
    """Ragged batches: records processed in place by one persistent launch
    (sbf_ragged_*; no reference counterpart).  Query output has one byte per
    window of the whole buffer; record r's hits are
    out[offset_r : offset_r + bytes_r - k + 1]."""

    def ragged_insert_async(self, d_seq, d_ranges, d_counts=None, stream=None) -> None:
        p, n = _dev_ptr(d_seq)
        rp, rn = _dev_ptr(d_ranges)
        cp = _dev_ptr(d_counts)[0] if d_counts is not None else None
        _check(_lib.sbf_ragged_insert_async(self._h, p, n, rp, rn // 16, cp, _stream(stream)))

    def ragged_contains_async(self, d_seq, d_ranges, d_out, d_counts=None, stream=None) -> None:
        p, n = _dev_ptr(d_seq)
        rp, rn = _dev_ptr(d_ranges)
        o, on = _dev_ptr(d_out)
        cp = _dev_ptr(d_counts)[0] if d_counts is not None else None
        _check(_lib.sbf_ragged_contains_async(self._h, p, n, rp, rn // 16, o, on, cp,
                                              _stream(stream)))

    def ragged_contains_counts_async(self, d_seq, d_ranges, d_record_valid, d_record_positive,
                                     d_out=None, d_counts=None, stream=None) -> None:
        """Ragged query with per-record valid / positive window counts
        computed in the query kernel (uint64 device arrays, one entry per
        record, zeroed by the call); `d_out` (hit bytes) is optional."""
        p, n = _dev_ptr(d_seq)
        rp, rn = _dev_ptr(d_ranges)
        vp, vn = _dev_ptr(d_record_valid)
        pp, pn = _dev_ptr(d_record_positive)
        if min(vn, pn) < (rn // 16) * 8:
            raise ValueError("per-record count arrays need one uint64 per record")
        o, on = _dev_ptr(d_out) if d_out is not None else (None, 0)
        cp = _dev_ptr(d_counts)[0] if d_counts is not None else None
        _check(_lib.sbf_ragged_contains_counts_async(self._h, p, n, rp, rn // 16, o, on, vp, pp,
                                                     cp, _stream(stream)))

    def ragged_insert(self, seq, ranges, tuning=None, stream=None) -> InsertReport:
        b = _host_bytes(seq)
        r = _ranges(ranges)
        rep = InsertReport()
        _check(_lib.sbf_ragged_insert(self._h, _np_ptr(b), b.size, _np_ptr(r), r.shape[0],
                                      _tuning(tuning), _stream(stream), C.byref(rep)))
        return rep

    def ragged_query_bits(self, seq, ranges, out=None, tuning=None, stream=None):
        """Returns (uint32 result words, QueryReport): window i -> bit i % 32
        of word i // 32."""
        b = _host_bytes(seq)
        r = _ranges(ranges)
        w = self.kmer_count(b.size)
        nw = (w + 31) // 32
        if out is None:
            out = np.zeros(max(nw, 1), np.uint32)
        o = out.numpy() if hasattr(out, "numpy") else out
        rep = QueryReport()
        _check(_lib.sbf_ragged_query_bits(self._h, _np_ptr(b), b.size, _np_ptr(r), r.shape[0],
                                          _np_ptr(o), o.nbytes // 4, _tuning(tuning),
                                          _stream(stream), C.byref(rep)))
        return o[:nw], rep

    def ragged_query(self, seq, ranges, out=None, tuning=None, stream=None):
        """Returns (hits, QueryReport); `out` may be a preallocated host array
        (pinned for the fastest copies) of at least len - k + 1 bytes."""
        b = _host_bytes(seq)
        r = _ranges(ranges)
        w = self.kmer_count(b.size)
        if out is None:
            out = np.zeros(max(w, 1), np.uint8)
        o = out.numpy() if hasattr(out, "numpy") else out
        rep = QueryReport()
        _check(_lib.sbf_ragged_query(self._h, _np_ptr(b), b.size, _np_ptr(r), r.shape[0],
                                     _np_ptr(o), o.size, _tuning(tuning), _stream(stream),
                                     C.byref(rep)))
        return o[:w], rep

    def ragged_autotune(self, seq, ranges, query: bool, sample_bytes: int = 0,
                        stream=None) -> RaggedTuning:
        b = _host_bytes(seq)
        r = _ranges(ranges)
        t = RaggedTuning()
        _check(_lib.sbf_ragged_autotune(self._h, int(query), _np_ptr(b), b.size, _np_ptr(r),
                                        r.shape[0], sample_bytes, _stream(stream), C.byref(t)))
        return t

    def ragged_tuning_lookup(self, nbytes: int, n_records: int, query: bool):
        """The tuning-table entry for a batch shape, or None."""
        t = RaggedTuning()
        st = _lib.sbf_ragged_tuning_lookup(self._h, int(query), nbytes, n_records, C.byref(t))
        return t if st == OK else None

    for f in (ragged_insert_async, ragged_contains_async, ragged_contains_counts_async,
              ragged_insert, ragged_query, ragged_query_bits, ragged_autotune,
              ragged_tuning_lookup):
        setattr(Filter, f.__name__, f)


_ragged_methods()


class _Reader:
    """Adapts bytes/str or a binary file-like object to the C read callback."""

    def __init__(self, source):
        import io

        if isinstance(source, str):
            source = source.encode()
        if isinstance(source, (bytes, bytearray, memoryview)):
            source = io.BytesIO(bytes(source))
        self.f = source
        self.error = None

        def _read(_user, buf, cap):
            try:
                data = self.f.read(cap)
            except Exception as e:  # surfaced as an io error
                self.error = e
                return -1
            if not data:
                return 0
            C.memmove(buf, data, len(data))
            return len(data)

        self.fn = READ_FN(_read)


def _fastx_view(v):
    hits = (np.ctypeslib.as_array(C.cast(v.hits, C.POINTER(C.c_uint8)), (v.n_hits,)).copy()
            if v.n_hits else np.zeros(0, np.uint8))
    return {"record_index": v.record_index,
            "header": C.string_at(v.header, v.header_bytes).decode(errors="replace")
            if v.header_bytes else "",
            "sequence": C.string_at(v.sequence, v.sequence_bytes) if v.sequence_bytes else b"",
            "queried_bases": v.queried_bases, "queried_kmers": v.queried_kmers,
            "positive_kmers": v.positive_kmers, "hits": hits}


def _consumer(consume, box):
    if consume is None:
        return FASTX_CB()

    def _cb(_user, vp):
        try:
            consume(_fastx_view(vp.contents))
            return 0
        except BaseException as e:  # noqa: BLE001 - re-raised after the call
            box.append(e)
            return 1
    return FASTX_CB(_cb)


def fastx_scan(source, source_name: str = "<stream>"):
    """FastxReader over `source` (bytes/str content, a binary file object, or
    a path via ``fastx_scan_file``): list of (header, sequence) pairs."""
    out = []

    def _cb(_u, _i, h, hn, s, sn):
        out.append((C.string_at(h, hn).decode(errors="replace") if hn else "",
                    C.string_at(s, sn) if sn else b""))
        return 0
    r = _Reader(source)
    cb = SCAN_CB(_cb)
    _check(_lib.sbf_fastx_scan(r.fn, None, source_name.encode(), cb, None, None))
    return out


def fastx_scan_file(path):
    out = []

    def _cb(_u, _i, h, hn, s, sn):
        out.append((C.string_at(h, hn).decode(errors="replace") if hn else "",
                    C.string_at(s, sn) if sn else b""))
        return 0
    cb = SCAN_CB(_cb)
    _check(_lib.sbf_fastx_scan_file(os.fsencode(path), cb, None, None))
    return out


def _fastx_methods():
    def insert_fastx(self, source, fill_fraction=0.7, stream=None, source_name="<stream>"):
        """insert_fastx (filter.cuh:416-421) over bytes/str or a binary file object."""
        r = _Reader(source)
        rep = InsertReport()
        _check(_lib.sbf_insert_fastx(self._h, r.fn, None, source_name.encode(), fill_fraction,
                                     _stream(stream), C.byref(rep)))
        return rep

    def insert_fastx_file(self, path, fill_fraction=0.7, stream=None):
        """insert_fastx_file (filter.cuh:437-452): plain or gzip file."""
        rep = InsertReport()
        _check(_lib.sbf_insert_fastx_file(self._h, os.fsencode(path), fill_fraction,
                                          _stream(stream), C.byref(rep)))
        return rep

    def query_fastx(self, source, fill_fraction=0.7, stream=None, source_name="<stream>",
                    consume=None):
        """query_fastx (filter.cuh:632-638); with `consume`, query_fastx_records."""
        r = _Reader(source)
        rep = QueryReport()
        box = []
        cb = _consumer(consume, box)
        st = _lib.sbf_query_fastx(self._h, r.fn, None, source_name.encode(), fill_fraction,
                                  _stream(stream), C.byref(rep), cb, None)
        if box:
            raise box[0]
        _check(st)
        return rep

    def query_fastx_file(self, path, fill_fraction=0.7, stream=None, consume=None):
        """query_fastx_file (filter.cuh:654-668); with `consume`,
        query_fastx_file_records (filter.cuh:713-735)."""
        rep = QueryReport()
        box = []
        cb = _consumer(consume, box)
        st = _lib.sbf_query_fastx_file(self._h, os.fsencode(path), fill_fraction, _stream(stream),
                                       C.byref(rep), cb, None)
        if box:
            raise box[0]
        _check(st)
        return rep

    def query_fastx_records(self, source, consume, fill_fraction=0.7, stream=None):
        return self.query_fastx(source, fill_fraction, stream, consume=consume)

    def query_fastx_file_records(self, path, consume, fill_fraction=0.7, stream=None):
        return self.query_fastx_file(path, fill_fraction, stream, consume=consume)

    def query_fastx_detailed(self, source, fill_fraction=0.7, stream=None):
        """query_fastx_detailed (filter.cuh:750-760): (summary, records)."""
        recs = []
        summary = self.query_fastx(source, fill_fraction, stream, consume=recs.append)
        return summary, recs

    def query_fastx_file_detailed(self, path, fill_fraction=0.7, stream=None):
        """query_fastx_file_detailed (filter.cuh:771-786)."""
        recs = []
        summary = self.query_fastx_file(path, fill_fraction, stream, consume=recs.append)
        return summary, recs

    for f in (insert_fastx, insert_fastx_file, query_fastx, query_fastx_file, query_fastx_records,
              query_fastx_file_records, query_fastx_detailed, query_fastx_file_detailed):
        setattr(Filter, f.__name__, f)


_fastx_methods()


_SYMBOL_WIDTH = {ALPHABET_DNA: 1, ALPHABET_PROTEIN: 1, ALPHABET_DNA_TRIPLET: 3}


def host_expand_threads() -> int:
    """Host threads that host-output queries expand bit-packed results with
    (0: they download one byte per window; SBF_HOST_EXPAND[_THREADS])."""
    return _lib.sbf_host_expand_threads()


def expand_result_bits(bits, n_windows: int, out=None, threads: int = 0) -> np.ndarray:
    """Bit-packed results (window i -> bit i % 32 of word i // 32) to one
    byte per window, on host threads (sbf_expand_result_bits)."""
    b = np.ascontiguousarray(np.asarray(bits).view(np.uint32).reshape(-1))
    if b.size * 32 < n_windows:
        raise ValueError("bit words hold fewer than n_windows results")
    o = np.empty(max(n_windows, 1), np.uint8) if out is None else out
    if o.size < n_windows:
        raise ValueError("output holds fewer than n_windows bytes")
    _check(_lib.sbf_expand_result_bits(_np_ptr(b), n_windows, _np_ptr(o), threads))
    return o[:n_windows]


def pack_dense_sequence(seq, alphabet: int = ALPHABET_DNA) -> np.ndarray:
    """Host dense packing (include/cusbf/dense_packed.hpp:36-50): one symbol
    per symbolWidth input bytes, 64 / symbolBits symbols per word."""
    b = _host_bytes(seq)
    n_sym = b.size // _SYMBOL_WIDTH[alphabet]
    n_words = _lib.sbf_dense_packed_word_count_for(alphabet, n_sym)
    out = np.zeros(max(n_words, 1), dtype=np.uint64)
    _check(_lib.sbf_pack_dense_host_for(alphabet, _np_ptr(b), n_sym, _np_ptr(out)))
    return out[:n_words]


def pack_dense_sequence_device(d_seq, num_symbols: int, d_words, stream=None,
                               alphabet: int = ALPHABET_DNA) -> None:
    """Device dense packing (include/cusbf/dense_packed.hpp:58-74)."""
    p, _ = _dev_ptr(d_seq)
    w, _ = _dev_ptr(d_words)
    if alphabet == ALPHABET_DNA:
        _check(_lib.sbf_pack_dense_device(p, num_symbols, w, _stream(stream)))
    else:
        _check(_lib.sbf_pack_dense_device_for(alphabet, p, num_symbols, w, _stream(stream)))


__all__ = [
    "Config", "Filter", "RecordRange", "InsertReport", "QueryReport", "SbfError",
    "NormalizedRecord", "QueryLayoutRecord", "normalize_record_batch", "query_layout",
    "normalized_batch_bytes", "validate_record_batch", "records_from_ranges",
    "fastx_scan", "fastx_scan_file",
    "pack_dense_sequence", "pack_dense_sequence_device", "lib", "version", "LIBRARY_PATH",
]


class Server:
    """Request server over a resident filter (sbf_server_*): continuous
    batching of insert and query requests from any number of threads; every
    result equals one-request-at-a-time execution in arrival order.  While it
    runs, the filter must not be used directly."""

    INSERT, QUERY, QUERY_BITS, QUERY_COUNTS = 0, 1, 2, 3
    # Flag for any op: `base` holds 2-bit dense-packed DNA words (32 symbols
    # per uint64) and `ranges` count symbols.
    DENSE = 0x10

    def __init__(self, filt: "Filter", **config):
        self._filter = filt
        cfg = ServerConfig(**config)
        h = _vp()
        _check(_lib.sbf_server_create(filt._h, C.byref(cfg), C.byref(h)))
        self._h = h
        self._refs: dict[int, tuple] = {}
        self._lock = threading.Lock()

    @staticmethod
    def now() -> float:
        return _lib.sbf_server_now()

    def submit_raw(self, op: int, base_ptr: int, ranges_ptr: int, n: int, out_ptr, out_len: int,
                   arrival: float = 0.0) -> int:
        """Pointer-level submit: the caller keeps the buffers alive."""
        t = _u64()
        _check(_lib.sbf_server_submit(self._h, op, base_ptr, ranges_ptr, n, out_ptr, out_len,
                                      arrival, C.byref(t)))
        return t.value

    def submit(self, op: int, base, ranges, out=None, arrival: float = 0.0) -> int:
        b = _host_bytes(base)
        r = _ranges(ranges)
        o = out
        bop = op & 0xF
        if bop != self.INSERT and o is None:
            span = max(int(r[-1, 0] + r[-1, 1]) - int(r[0, 0]), 0) if r.shape[0] else 0
            w = max(span - self._filter.config.k + 1, 0)
            if bop == self.QUERY:
                o = np.zeros(max(w, 1), np.uint8)
            elif bop == self.QUERY_COUNTS:
                o = np.zeros((max(r.shape[0], 1), 2), np.uint64)
            else:
                o = np.zeros(max((w + 31) // 32, 1), np.uint32)
        t = self.submit_raw(op, _np_ptr(b), _np_ptr(r), r.shape[0],
                            _np_ptr(o) if o is not None else None,
                            o.nbytes if o is not None else 0, arrival)
        with self._lock:
            self._refs[t] = (b, r, o)
        return t

    def submit_query(self, base, ranges, out=None, arrival: float = 0.0) -> int:
        return self.submit(self.QUERY, base, ranges, out, arrival)

    def submit_insert(self, base, ranges, arrival: float = 0.0) -> int:
        return self.submit(self.INSERT, base, ranges, None, arrival)

    def wait(self, ticket: int, timeout: float = 0.0):
        """Waits for a request; returns (info dict, result or None): hit
        bytes (QUERY), bit words (QUERY_BITS), or an (n, 2) array of
        per-record (valid, positive) windows (QUERY_COUNTS)."""
        info = ServerRequestInfo()
        st = _lib.sbf_server_wait(self._h, ticket, timeout, C.byref(info))
        with self._lock:
            refs = self._refs.pop(ticket, None)
        _check(st)
        out = None
        if refs is not None and refs[2] is not None:
            o = refs[2]
            if o.dtype == np.uint8:
                out = o[:info.windows]
            elif o.dtype == np.uint64:
                out = o.reshape(-1, 2)[:refs[1].shape[0]]
            else:
                out = o[:(info.windows + 31) // 32]
        return info.as_dict(), out

    def drain(self) -> None:
        _check(_lib.sbf_server_drain(self._h))

    def stats(self, reset: bool = False) -> dict:
        s = ServerStats()
        _check(_lib.sbf_server_get_stats(self._h, int(reset), C.byref(s)))
        return s.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.sbf_server_destroy(self._h)
            self._h = None
            self._refs.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

