"""Build ``fhs_b200/libfhs_b200.so`` for sm_100a with nvcc (in-tree), and the
standalone C harness ``fhs_b200/fhs_harness`` over its C ABI (gcc).

Usage: ``python faceted-hypersara_b200/build.py [--force]``.  Objects go to
``faceted-hypersara_b200/_build/`` (git-ignored); the shared library is
written next to the Python package so that it travels with the tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "fhs_b200", "libfhs_b200.so")
HARNESS = os.path.join(HERE, "fhs_b200", "fhs_harness")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def build(force: bool = False, verbose: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    hdr_mtime = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_mtime):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [nvcc, *NVCC_FLAGS, "-x", "c++", "-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for err in ex.map(run, jobs):
            if verbose and err:
                print(err)
    if jobs or force or not os.path.exists(OUT):
        cmd = [nvcc, *ARCH, "-shared", "-o", OUT, *objs, "-lcufft", "-lcudart"]
        run(cmd)
    # the standalone C harness (plain C99 over the C ABI), next to the library
    hsrc = os.path.join(HERE, "harness", "fhs_harness.c")
    if force or not os.path.exists(HARNESS) or os.path.getmtime(HARNESS) < max(
            os.path.getmtime(hsrc), os.path.getmtime(OUT), hdr_mtime):
        cc = shutil.which("gcc") or shutil.which("cc")
        if cc is None:
            raise RuntimeError("no C compiler for the harness")
        run([cc, "-O2", "-std=c99", "-D_POSIX_C_SOURCE=200809L", "-Wall", "-I", INCLUDE, hsrc,
             "-L", os.path.dirname(OUT), "-lfhs_b200", "-Wl,-rpath,$ORIGIN", "-lm", "-o", HARNESS])
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
