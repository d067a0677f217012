"""The C-ABI library loads and exports every symbol its headers declare (CPU).

No compute runs here: without a GPU, sbf_filter_create must fail loudly with
a CUDA error (there is no CPU fallback), while pure host helpers work.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(sbf_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    # typedef'd callback types are not exported symbols
    return sorted(n for n in names if not n.endswith("_cb") and not n.endswith("_fn"))


def test_library_exports_all_declared_symbols(sbf):
    lib = ctypes.CDLL(sbf.LIBRARY_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", sbf.LIBRARY_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (sbf_[a-z0-9_]+)$", out, flags=re.M))
    assert set(names) <= exported


def test_no_cpu_fallback_without_gpu(sbf):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible; the CPU-only behaviour is not observable here")
    with pytest.raises(sbf.SbfError) as e:
        sbf.Filter(1 << 12)
    assert e.value.category == "cuda"


def test_host_helpers(sbf, oracle_mod):
    o = oracle_mod.Oracle()
    rng = np.random.default_rng(1)
    seq = rng.choice(np.frombuffer(b"ACGTNacgt", np.uint8), 1001)
    np.testing.assert_array_equal(sbf.pack_dense_sequence(seq), o.pack_dense(seq))
    assert sbf.Filter.dense_packed_word_count(0) == 0
    assert sbf.Filter.dense_packed_word_count(32) == 1
    assert sbf.Filter.dense_packed_word_count(33) == 2
    assert sbf.version().startswith("sbf-b200")
