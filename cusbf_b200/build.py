"""Builds libsbf_b200.so in-tree with nvcc for sm_100a.

``python cusbf_b200/build.py`` compiles the
CUDA sources in cusbf_b200/csrc/ into cusbf_b200/libsbf_b200.so.  The build
is incremental: it is skipped when the library is newer than every source.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsbf_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


# The tile kernel source, embedded for run-time compilation (sbf_jit.cpp).
JIT_SOURCES = [("kJitInternal", "sbf_internal.h"), ("kJitDevice", "sbf_device.cuh"),
               ("kJitFlush", "sbf_flush.cuh"), ("kJitTile", "sbf_tile.cuh"),
               ("kJitGeneric", "sbf_generic.cuh")]


def write_jit_sources(objdir: str) -> None:
    out = []
    for var, name in JIT_SOURCES:
        text = open(os.path.join(CSRC, name)).read()
        if ")SBFJIT\"" in text:
            raise RuntimeError(f"{name} contains the raw-string delimiter")
        out.append(f'static const char {var}[] = R"SBFJIT({text})SBFJIT";\n')
    path = os.path.join(objdir, "sbf_jit_sources.inc")
    data = "".join(out)
    if not os.path.exists(path) or open(path).read() != data:
        with open(path, "w") as fh:
            fh.write(data)


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = sources()
    if not force and not _stale(LIB, srcs + headers() + [__file__]):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    write_jit_sources(objdir)
    objs = []
    procs = []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [NVCC, *ARCH_FLAGS, *COMMON, "-I", os.path.join(ROOT, "include"), "-I", objdir,
               "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB + ".tmp"
    link = [NVCC, *ARCH_FLAGS, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs, "-lz", "-ldl"]
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
