"""ctypes bindings for the CPU oracle and the reference-backed checkers.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check in
__graft_entry__.py and by the CPU-baseline leg of bench.py.  The product
(cusbf_b200) never imports this module.

* ``Oracle``  -- oracle/_build/libsbf_oracle.so, the C restatement of the
  reference semantics (oracle/sbf_oracle.c).
* ``RefCpu``  -- oracle/_ref/libsbf_refcpu.so, the reference cuSBF's own
  host-callable arithmetic driven window by window (oracle/ref_cpu.cu).
* ``RefGpu``  -- oracle/_ref/libsbf_refgpu.so, the unmodified reference GPU
  filter compiled for sm_100a (oracle/ref_gpu.cu).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libsbf_oracle.so")
REFCPU_SO = os.path.join(HERE, "_ref", "libsbf_refcpu.so")
REFGPU_SO = os.path.join(HERE, "_ref", "libsbf_refgpu.so")

ALPHABET_DNA = 0
ALPHABET_DNA_TRIPLET = 1
ALPHABET_PROTEIN = 2

# Configuration ids understood by oracle/ref_cpu.cu.
REF_CONFIGS = {
    (31, 28, 16, 4, ALPHABET_DNA): 0,
    (5, 4, 3, 4, ALPHABET_DNA): 1,
    (5, 4, 3, 4, ALPHABET_PROTEIN): 2,
    (3, 2, 2, 4, ALPHABET_DNA_TRIPLET): 3,
    (31, 28, 16, 8, ALPHABET_DNA): 4,
    (31, 28, 16, 16, ALPHABET_DNA): 5,
    (21, 19, 11, 4, ALPHABET_DNA): 6,
}


class _Cfg(C.Structure):
    _fields_ = [
        ("k", C.c_uint32),
        ("s", C.c_uint32),
        ("m", C.c_uint32),
        ("hashes", C.c_uint32),
        ("alphabet", C.c_int32),
    ]


def build_oracle() -> None:
    """Compiles the oracle (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _as_bytes(seq) -> np.ndarray:
    if isinstance(seq, np.ndarray):
        return np.ascontiguousarray(seq, dtype=np.uint8)
    if isinstance(seq, str):
        seq = seq.encode()
    return np.frombuffer(bytes(seq), dtype=np.uint8)


def num_shards(requested_bits: int) -> int:
    blocks = max(1, (requested_bits + 255) // 256)
    p = 1
    while p < blocks:
        p <<= 1
    return p


def symbol_params(alphabet: int) -> tuple[int, int]:
    return {ALPHABET_DNA: (2, 1), ALPHABET_DNA_TRIPLET: (6, 3), ALPHABET_PROTEIN: (5, 1)}[alphabet]


def windows(k: int, nbytes: int, alphabet: int = ALPHABET_DNA) -> int:
    _, width = symbol_params(alphabet)
    n = nbytes // width
    return 0 if n < k else n - k + 1


class Oracle:
    """The C restatement; every call takes the k,s,m,hashes of the filter."""

    def __init__(self, k=31, s=28, m=16, hashes=4, alphabet=ALPHABET_DNA, threads=None):
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        self.lib = C.CDLL(ORACLE_SO)
        self.cfg = _Cfg(k, s, m, hashes, alphabet)
        self.k, self.s, self.m, self.hashes, self.alphabet = k, s, m, hashes, alphabet
        self.threads = threads or os.cpu_count() or 1
        L = self.lib
        for name in ("sbf_oracle_insert", "sbf_oracle_contains", "sbf_oracle_pack_dense",
                     "sbf_oracle_insert_dense", "sbf_oracle_contains_dense",
                     "sbf_oracle_window_shards", "sbf_oracle_count_runs", "sbf_oracle_runs"):
            getattr(L, name).restype = C.c_int
        L.sbf_oracle_hash64.restype = C.c_uint64
        L.sbf_oracle_hash64.argtypes = [C.c_uint64]
        L.sbf_oracle_minimizer_hash64.restype = C.c_uint64
        L.sbf_oracle_minimizer_hash64.argtypes = [C.c_uint64]

    def new_words(self, requested_bits: int) -> np.ndarray:
        return np.zeros(num_shards(requested_bits) * 4, dtype=np.uint64)

    def insert(self, words: np.ndarray, seq, threads=None) -> int:
        b = _as_bytes(seq)
        out = C.c_uint64(0)
        rc = self.lib.sbf_oracle_insert(C.byref(self.cfg), _ptr(b), C.c_uint64(b.size),
                                        _ptr(words), C.c_uint64(words.size // 4),
                                        C.c_int(threads or self.threads), C.byref(out))
        if rc != 0:
            raise ValueError(f"oracle insert failed ({rc})")
        return out.value

    def contains(self, words: np.ndarray, seq, threads=None) -> np.ndarray:
        b = _as_bytes(seq)
        n = windows(self.k, b.size, self.alphabet)
        out = np.zeros(max(n, 1), dtype=np.uint8)
        rc = self.lib.sbf_oracle_contains(C.byref(self.cfg), _ptr(b), C.c_uint64(b.size),
                                          _ptr(words), C.c_uint64(words.size // 4), _ptr(out),
                                          C.c_int(threads or self.threads))
        if rc != 0:
            raise ValueError(f"oracle contains failed ({rc})")
        return out[:n]

    def pack_dense(self, seq) -> np.ndarray:
        b = _as_bytes(seq)
        bits, width = symbol_params(self.alphabet)
        n = b.size // width
        per = 64 // bits
        out = np.zeros(max((n + per - 1) // per, 1), dtype=np.uint64)
        self.lib.sbf_oracle_pack_dense(C.byref(self.cfg), _ptr(b), C.c_uint64(b.size), _ptr(out))
        return out[: (n + per - 1) // per]

    def insert_dense(self, words, packed, num_symbols, threads=None):
        packed = np.ascontiguousarray(packed, dtype=np.uint64)
        self.lib.sbf_oracle_insert_dense(C.byref(self.cfg), _ptr(packed), C.c_uint64(num_symbols),
                                         _ptr(words), C.c_uint64(words.size // 4),
                                         C.c_int(threads or self.threads))

    def contains_dense(self, words, packed, num_symbols, threads=None):
        packed = np.ascontiguousarray(packed, dtype=np.uint64)
        n = 0 if num_symbols < self.k else num_symbols - self.k + 1
        out = np.zeros(max(n, 1), dtype=np.uint8)
        self.lib.sbf_oracle_contains_dense(C.byref(self.cfg), _ptr(packed),
                                           C.c_uint64(num_symbols), _ptr(words),
                                           C.c_uint64(words.size // 4), _ptr(out),
                                           C.c_int(threads or self.threads))
        return out[:n]

    def window_shards(self, seq, n_shards):
        b = _as_bytes(seq)
        n = windows(self.k, b.size, self.alphabet)
        shards = np.zeros(max(n, 1), dtype=np.uint32)
        valid = np.zeros(max(n, 1), dtype=np.uint8)
        self.lib.sbf_oracle_window_shards(C.byref(self.cfg), _ptr(b), C.c_uint64(b.size),
                                          C.c_uint64(n_shards), _ptr(shards), _ptr(valid))
        return shards[:n], valid[:n]

    def runs(self, seq, n_shards) -> tuple[np.ndarray, np.ndarray]:
        """Run records of ``seq``: (shards uint32[R], masks uint64[R, 4]); ORing
        every record's masks into its shard of an empty filter gives the
        filter that ``insert`` builds."""
        b = _as_bytes(seq)
        cap = max(windows(self.k, b.size, self.alphabet), 1)
        shards = np.zeros(cap, dtype=np.uint32)
        masks = np.zeros((cap, 4), dtype=np.uint64)
        n = C.c_uint64(0)
        rc = self.lib.sbf_oracle_runs(C.byref(self.cfg), _ptr(b), C.c_uint64(b.size),
                                      C.c_uint64(n_shards), _ptr(shards), _ptr(masks),
                                      C.c_uint64(cap), C.byref(n))
        if rc != 0:
            raise RuntimeError(f"sbf_oracle_runs failed ({rc})")
        return shards[:n.value].copy(), masks[:n.value].copy()

    def count_runs(self, seq, n_shards) -> tuple[int, int]:
        """Super-k-mer runs R and valid windows of ``seq`` for a filter with
        ``n_shards`` shards (the R of the algorithmic-bytes model)."""
        b = _as_bytes(seq)
        runs, valid = C.c_uint64(0), C.c_uint64(0)
        self.lib.sbf_oracle_count_runs(C.byref(self.cfg), _ptr(b), C.c_uint64(b.size),
                                       C.c_uint64(n_shards), C.byref(runs), C.byref(valid))
        return runs.value, valid.value


class RefCpu:
    """The reference's own arithmetic on the CPU (oracle/_ref, built here)."""

    def __init__(self, k=31, s=28, m=16, hashes=4, alphabet=ALPHABET_DNA, threads=None):
        if not os.path.exists(REFCPU_SO):
            raise FileNotFoundError(REFCPU_SO)
        self.lib = C.CDLL(REFCPU_SO)
        self.cfg_id = REF_CONFIGS[(k, s, m, hashes, alphabet)]
        self.k, self.alphabet = k, alphabet
        self.threads = threads or os.cpu_count() or 1

    @staticmethod
    def available() -> bool:
        return os.path.exists(REFCPU_SO)

    def insert(self, words, seq, threads=None):
        b = _as_bytes(seq)
        rc = self.lib.sbf_refcpu_insert(C.c_int(self.cfg_id), _ptr(b), C.c_uint64(b.size),
                                        _ptr(words), C.c_uint64(words.size // 4),
                                        C.c_int(threads or self.threads))
        assert rc == 0

    def contains(self, words, seq, threads=None):
        b = _as_bytes(seq)
        n = windows(self.k, b.size, self.alphabet)
        out = np.zeros(max(n, 1), dtype=np.uint8)
        rc = self.lib.sbf_refcpu_contains(C.c_int(self.cfg_id), _ptr(b), C.c_uint64(b.size),
                                          _ptr(words), C.c_uint64(words.size // 4), _ptr(out),
                                          C.c_int(threads or self.threads))
        assert rc == 0
        return out[:n]

    def insert_dense(self, words, packed, num_symbols, threads=None):
        packed = np.ascontiguousarray(packed, dtype=np.uint64)
        rc = self.lib.sbf_refcpu_insert_dense(C.c_int(self.cfg_id), _ptr(packed),
                                              C.c_uint64(num_symbols), _ptr(words),
                                              C.c_uint64(words.size // 4),
                                              C.c_int(threads or self.threads))
        assert rc == 0


class RefGpu:
    """Handle over the unmodified reference GPU filter (oracle/_ref)."""

    def __init__(self, requested_bits, cfg_id=0):
        if not os.path.exists(REFGPU_SO):
            raise FileNotFoundError(REFGPU_SO)
        L = C.CDLL(REFGPU_SO)
        self.lib = L
        L.sbf_refgpu_create.restype = C.c_void_p
        L.sbf_refgpu_create.argtypes = [C.c_int, C.c_uint64]
        L.sbf_refgpu_destroy.argtypes = [C.c_void_p]
        L.sbf_refgpu_clear.argtypes = [C.c_void_p, C.c_void_p]
        L.sbf_refgpu_insert_async.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        L.sbf_refgpu_contains_async.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                                C.c_uint64, C.c_void_p]
        L.sbf_refgpu_words.restype = C.c_void_p
        L.sbf_refgpu_words.argtypes = [C.c_void_p]
        L.sbf_refgpu_num_shards.restype = C.c_uint64
        L.sbf_refgpu_num_shards.argtypes = [C.c_void_p]
        self.h = L.sbf_refgpu_create(cfg_id, requested_bits)
        if not self.h:
            raise RuntimeError("reference filter construction failed")

    @staticmethod
    def available() -> bool:
        return os.path.exists(REFGPU_SO)

    def close(self):
        if self.h:
            self.lib.sbf_refgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def num_shards(self) -> int:
        return self.lib.sbf_refgpu_num_shards(self.h)

    def words_ptr(self) -> int:
        return self.lib.sbf_refgpu_words(self.h)

    def clear(self, stream=0):
        assert self.lib.sbf_refgpu_clear(self.h, C.c_void_p(stream)) == 0

    def insert_async(self, d_ptr, nbytes, stream=0):
        assert self.lib.sbf_refgpu_insert_async(self.h, C.c_void_p(d_ptr), nbytes,
                                                C.c_void_p(stream)) == 0

    def contains_async(self, d_ptr, nbytes, d_out, out_len, stream=0):
        assert self.lib.sbf_refgpu_contains_async(self.h, C.c_void_p(d_ptr), nbytes,
                                                  C.c_void_p(d_out), out_len,
                                                  C.c_void_p(stream)) == 0
