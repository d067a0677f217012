"""DNA configurations that are not compiled into the library run the same
tile kernels compiled at run time (sbf_jit.cpp, NVRTC): bit-identical to the
oracle and to the generic kernels through the sequence, dense, ragged,
record-batch and server paths, with the compiled cubin cached on disk."""
import os

import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu

CONFIGS = [dict(k=25, s=22, m=13, hashes=4), dict(k=17, s=15, m=9, hashes=8),
           dict(k=32, s=32, m=32, hashes=12), dict(k=1, s=1, m=1, hashes=16)]
IDS = ["k25", "k17h8", "k32h12", "k1h16"]


@pytest.fixture(scope="module")
def jit_cache(tmp_path_factory):
    d = tmp_path_factory.mktemp("jit_cache")
    old = os.environ.get("SBF_JIT_CACHE")
    os.environ["SBF_JIT_CACHE"] = str(d)
    os.environ.pop("SBF_JIT", None)
    yield d
    if old is None:
        os.environ.pop("SBF_JIT_CACHE", None)
    else:
        os.environ["SBF_JIT_CACHE"] = old


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_runtime_compiled_match_oracle(sbf, cuda, oracle_mod, jit_cache, monkeypatch, cfg):
    torch = cuda
    rng = np.random.default_rng(cfg["k"] + cfg["hashes"])
    ins = random_dna(rng, 200_000, b"ACGTACGTACGTACGTacgtN")
    qry = np.concatenate([ins[:50_000], random_dna(rng, 50_000)])
    bits = 1 << 18
    o = oracle_mod.Oracle(**cfg)
    w = o.new_words(bits)
    o.insert(w, ins)
    want = o.contains(w, qry)
    f = sbf.Filter(bits, **cfg)
    assert f.kernel_path() == sbf.Filter.KERNELS_RUNTIME_COMPILED
    f.insert_sequence(ins)
    np.testing.assert_array_equal(f.words_host(), w)
    np.testing.assert_array_equal(f.contains_sequence(qry), want)
    # misaligned device buffers (grid phase) and bit-packed results
    d_q = torch.from_numpy(np.concatenate([np.zeros(5, np.uint8), qry])).cuda()[5:]
    out = torch.zeros(want.size + 3, dtype=torch.uint8, device="cuda")
    f.contains_sequence_async(d_q, out[3:])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out[3:].cpu().numpy(), want)
    bits_out = f.contains_sequence_bits(qry)
    packed = np.packbits(want, bitorder="little")
    packed = np.concatenate([packed, np.zeros(bits_out.size * 4 - packed.size, np.uint8)])
    np.testing.assert_array_equal(bits_out.view(np.uint8), packed)
    # dense input
    dense = sbf.pack_dense_sequence(ins)
    g = sbf.Filter(bits, **cfg)
    g.insert_dense_packed(dense, ins.size)
    w2 = o.new_words(bits)
    o.insert_dense(w2, dense, ins.size)
    np.testing.assert_array_equal(g.words_host(), w2)
    np.testing.assert_array_equal(g.contains_dense_packed(dense, ins.size),
                                  o.contains_dense(w2, dense, ins.size))
    # the generic kernels give the same words
    monkeypatch.setenv("SBF_JIT", "0")
    h = sbf.Filter(bits, **cfg)
    assert h.kernel_path() == sbf.Filter.KERNELS_GENERIC
    h.insert_sequence(ins)
    np.testing.assert_array_equal(h.words_host(), w)
    assert any(p.name.startswith(f"tile_k{cfg['k']}_s{cfg['s']}_m{cfg['m']}_h{cfg['hashes']}_")
               for p in jit_cache.iterdir())


def test_runtime_compiled_ragged_records_server(sbf, cuda, oracle_mod, jit_cache):
    cfg = CONFIGS[0]
    k = cfg["k"]
    rng = np.random.default_rng(99)
    parts, ranges, pos = [], [], 0
    for i in range(400):
        if rng.random() < 0.3:
            parts.append(random_dna(rng, 7))
            pos += 7
        n = int(rng.integers(0, 500))
        parts.append(random_dna(rng, n, b"ACGTACGTACGTN"))
        ranges.append((pos, n))
        pos += n
    seq = np.concatenate(parts)
    o = oracle_mod.Oracle(**cfg)
    bits = 1 << 18
    f = sbf.Filter(bits, **cfg)
    assert f.kernel_path() == sbf.Filter.KERNELS_RUNTIME_COMPILED
    f.ragged_insert(seq, ranges[::2])
    w = o.new_words(bits)
    for off, n in ranges[::2]:
        o.insert(w, seq[off:off + n])
    np.testing.assert_array_equal(f.words_host(), w)
    hits, rep = f.ragged_query(seq, ranges, tuning=dict(chunk_bytes=8192, stages=2,
                                                        ctas_per_sm=0, use_graph=1))
    pos_total = 0
    for off, n in ranges:
        if n >= k:
            want = o.contains(w, seq[off:off + n])
            np.testing.assert_array_equal(hits[off:off + n - k + 1], want)
            pos_total += int(want.sum())
    assert rep.positive_kmers == pos_total
    recs = []
    f.query_record_batch(seq, ranges, consume=recs.append)
    assert sum(r["positive_kmers"] for r in recs) == pos_total
    srv = sbf.Server(f, staging_bytes=1 << 26, pinned_bytes=1 << 24, use_graph=1)
    r = np.asarray(ranges[:50], np.uint64)
    t = srv.submit(sbf.Server.QUERY, seq, r)
    _, got = srv.wait(t, timeout=60.0)
    lo, hi = int(r[0, 0]), int(r[-1, 0] + r[-1, 1])
    np.testing.assert_array_equal(got, hits[lo:hi - k + 1])
    srv.close()


def test_runtime_compilation_with_another_nvrtc_loaded(tmp_path):
    """A process that already holds an older libnvrtc.so.12 (Python frameworks
    ship one) still compiles with the toolkit's NVRTC."""
    import glob
    import subprocess
    import sys

    import torch

    cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_nvrtc",
                                   "lib", "libnvrtc.so*"))
    if not cands:
        pytest.skip("no second libnvrtc in this environment")
    code = f"""
import ctypes, os, sys
ctypes.CDLL({cands[0]!r}, mode=ctypes.RTLD_GLOBAL)
sys.path.insert(0, {os.path.dirname(os.path.dirname(os.path.abspath(__file__)))!r})
import cusbf_b200 as sbf
f = sbf.Filter(1 << 16, k=23, s=21, m=12, hashes=4)
print(f.kernel_path())
"""
    env = dict(os.environ, SBF_JIT_CACHE=str(tmp_path))
    env.pop("SBF_JIT", None)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip().splitlines()[-1] == "1", r.stdout + r.stderr


ALPHA_CONFIGS = [dict(k=12, s=10, m=6, hashes=4, alphabet=2), dict(k=5, s=4, m=3, hashes=8, alphabet=2),
                 dict(k=10, s=8, m=5, hashes=16, alphabet=1), dict(k=3, s=2, m=2, hashes=4, alphabet=1)]


@pytest.mark.parametrize("cfg", ALPHA_CONFIGS, ids=["prot12", "prot5h8", "trip10h16", "trip3"])
def test_runtime_compiled_alphabets_match_oracle(sbf, cuda, oracle_mod, jit_cache, cfg):
    """Protein and DNA-triplet configurations run the generic kernels compiled
    with the configuration as constants."""
    rng = np.random.default_rng(cfg["k"] * 3 + cfg["alphabet"])
    if cfg["alphabet"] == 2:
        a = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWYacdefghiklmnpqrstvwy*X-", np.uint8)
        ins = a[rng.integers(0, a.size, 150_000)]
        qry = np.concatenate([ins[:40_000], a[rng.integers(0, a.size, 40_000)]])
        width = 1
    else:
        ins = random_dna(rng, 150_001, b"ACGTACGTACGTacgtN")
        qry = np.concatenate([ins[:60_000], random_dna(rng, 60_000)])
        width = 3
    bits = 1 << 17
    o = oracle_mod.Oracle(**cfg)
    w = o.new_words(bits)
    o.insert(w, ins)
    want = o.contains(w, qry)
    f = sbf.Filter(bits, **cfg)
    assert f.kernel_path() == sbf.Filter.KERNELS_RUNTIME_COMPILED
    f.insert_sequence(ins)
    np.testing.assert_array_equal(f.words_host(), w)
    np.testing.assert_array_equal(f.contains_sequence(qry), want)
    packed = sbf.pack_dense_sequence(qry, alphabet=cfg["alphabet"])
    n_sym = qry.size // width
    np.testing.assert_array_equal(f.contains_dense_packed(packed, n_sym),
                                  o.contains_dense(w, packed, n_sym))
    # record batches (symbol-aligned ranges) with per-record counts
    ranges = [(i * 30 * width, 25 * width) for i in range(qry.size // (30 * width))]
    recs = []
    f.query_record_batch(qry, ranges, consume=recs.append)
    for (off, n), r in zip(ranges, recs):
        np.testing.assert_array_equal(r["hits"], o.contains(w, qry[off:off + n]))
