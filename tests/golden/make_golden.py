"""Generates the golden parity fixtures in tests/golden/.

The expected values come from oracle/_ref/libsbf_refcpu.so: the reference
cuSBF's own host-callable arithmetic (Alphabet encode, extractPackedSubwindow,
minimizer_hash64, hash64, filter_block::sectorizedBitAddress) compiled from
the reference headers by oracle/Makefile and driven window by window
(oracle/ref_cpu.cu).  Inputs are seeded, so the fixtures can be regenerated:

    make -C oracle && python tests/golden/make_golden.py

Outputs:
  * k31_small.npz   -- full word arrays and query bytes for small inputs
                       (k=31,s=28,m=16,h=4, the other compiled configs, and
                       the protein and DNA-triplet alphabets).
  * digests.json    -- SHA-256 digests of the word arrays and query bytes of
                       the plain-method small workload (2 Mbp, 85.7 bits per
                       k-mer, + a fresh 2 Mbp query record) and of a 20 Mbp
                       genome-like case; checked on the GPU without the oracle.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import RefCpu, num_shards, windows  # noqa: E402

SMALL_CASES = [
    # (name, k, s, m, h, bits, insert_len, seed, alphabet-bytes)
    ("k31_uniform", 31, 28, 16, 4, 1 << 16, 20_000, 42, b"ACGT"),
    ("k31_invalid", 31, 28, 16, 4, 1 << 14, 20_000, 43, b"ACGTACGTACGTacgtN"),
    ("k31_h8", 31, 28, 16, 8, 1 << 16, 10_000, 44, b"ACGT"),
    ("k31_h16", 31, 28, 16, 16, 1 << 16, 10_000, 45, b"ACGT"),
    ("k21", 21, 19, 11, 4, 1 << 15, 10_000, 46, b"ACGTN"),
    ("k5", 5, 4, 3, 4, 1 << 12, 2_000, 47, b"ACGT"),
]
# Protein and DNA-triplet alphabets (alphabet id, as in the C ABI):
# (name, k, s, m, h, bits, insert_len, seed, letters, alphabet)
ALPHABET_CASES = [
    ("prot5", 5, 4, 3, 4, 1 << 12, 3_000, 48, b"ACDEFGHIKLMNPQRSTVWYacdefXB*", 2),
    ("trip3", 3, 2, 2, 4, 1 << 12, 6_000, 49, b"ACGTACGTACGTacgtN", 1),
]


def seq_of(rng, n, alphabet):
    a = np.frombuffer(alphabet, dtype=np.uint8)
    return a[rng.integers(0, len(a), size=n)]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def plain_small_inputs():
    """The plain-method small workload: one 2 Mbp uniform ACGT record (seed
    42), queried with itself plus a fresh 2 Mbp record (seed 1337)."""
    from workloads.synthetic import uniform_dna

    ins = uniform_dna(2_000_000, seed=42)
    fresh = uniform_dna(2_000_000, seed=1337)
    return ins, fresh


def main() -> None:
    arrays = {}
    cases = [c + (0,) for c in SMALL_CASES] + ALPHABET_CASES
    for name, k, s, m, h, bits, n, seed, alpha, alphabet in cases:
        rng = np.random.default_rng(seed)
        ins = seq_of(rng, n, alpha)
        qry = np.concatenate([ins[: n // 2], seq_of(rng, n, alpha)])
        r = RefCpu(k, s, m, h, alphabet)
        w = np.zeros(num_shards(bits) * 4, dtype=np.uint64)
        r.insert(w, ins)
        hits = r.contains(w, qry)
        arrays[f"{name}__insert"] = ins
        arrays[f"{name}__query"] = qry
        arrays[f"{name}__words"] = w
        arrays[f"{name}__hits"] = hits
        arrays[f"{name}__cfg"] = np.array([k, s, m, h, bits], dtype=np.uint64)
        arrays[f"{name}__alphabet"] = np.array([alphabet], dtype=np.uint64)
    np.savez_compressed(os.path.join(HERE, "k31_small.npz"), **arrays)

    digests = {}
    ins, fresh = plain_small_inputs()
    n_ins = windows(31, ins.size)
    bits = int(round(85.7 * n_ins))
    r = RefCpu()
    w = np.zeros(num_shards(bits) * 4, dtype=np.uint64)
    r.insert(w, ins)
    qry_pos = r.contains(w, ins)
    qry_neg = r.contains(w, fresh)
    digests["plain_small"] = {
        "requested_bits": bits,
        "num_shards": num_shards(bits),
        "insert_seed": 42,
        "fresh_seed": 1337,
        "words_sha256": sha(w),
        "hits_positive_sha256": sha(qry_pos),
        "hits_fresh_sha256": sha(qry_neg),
        "positives": int(qry_pos.sum()),
        "false_positives": int(qry_neg.sum()),
        "set_bits": int(np.unpackbits(w.view(np.uint8)).sum()),
    }

    from workloads.synthetic import genome_records, join_records

    recs = genome_records(total_bp=20_000_000, n_records=3, seed=7, gc=0.36,
                          tandem_frac=0.03, n_run_frac=0.001)
    joined, _ = join_records(recs)
    bits = 1 << 26
    w = np.zeros(num_shards(bits) * 4, dtype=np.uint64)
    r.insert(w, joined)
    hits = r.contains(w, joined[::-1].copy())
    digests["genome_20m"] = {
        "requested_bits": bits,
        "seed": 7,
        "words_sha256": sha(w),
        "hits_reversed_sha256": sha(hits),
        "positives_reversed": int(hits.sum()),
        "joined_sha256": sha(joined),
    }
    with open(os.path.join(HERE, "digests.json"), "w") as fh:
        json.dump(digests, fh, indent=1)
    print(json.dumps(digests, indent=1))


if __name__ == "__main__":
    main()
