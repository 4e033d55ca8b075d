"""Builds libmdx.so (the CUDA hot path + C ABI) in-tree for sm_100a.

Each csrc/*.cu is compiled to an object under md_engine_b200/_build/ (in
parallel, skipped when up to date) and linked with cuFFT into
md_engine_b200/libmdx.so.  No PyTorch types cross the ABI; PyTorch is not
needed to build or to load the library.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmdx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "mdx.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src, extra, verbose):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    path = os.path.join(CSRC, src)
    hm = _headers_mtime()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), hm):
        return obj, ""
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, (r.stderr if verbose else "")


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, verbose or ptxas_info), srcs))
    objs = [o for o, _ in results]
    logs = "".join(l for _, l in results)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcufft", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return logs


if __name__ == "__main__":
    out = build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    if out:
        print(out)
    print(LIB)
