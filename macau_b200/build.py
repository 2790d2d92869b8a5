"""Builds the in-tree CUDA library macau_b200/_lib/libmacau_b200.so for sm_100a.

Every translation unit under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` (in parallel) and linked into one
shared library that exports the C ABI of include/macau_b200.h.  IEEE arithmetic is kept (no
fast-math): the FP64 path is compared with the FP64 oracle at 1e-9.

    python -m macau_b200.build [--verbose] [--ptxas]
"""
import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libmacau_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler():
    # nvcc's default host compiler is `g++` on PATH; prefer the system one explicitly.
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else shutil.which("g++")


def _flags(ptxas):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                "-ccbin", host_compiler(), f"-I{ROOT / 'include'}", "--expt-relaxed-constexpr",
                "-Xcudafe", "--diag_suppress=177"]
    if ptxas:
        f += ["-Xptxas", "-v"]
    return f


def _compile(src, ptxas, verbose):
    obj = OBJ / (src.stem + ".o")
    deps = [src] + sorted(SRC.glob("*.cuh")) + sorted(SRC.glob("*.h")) + [ROOT / "include" / "macau_b200.h"]
    if obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps) and not ptxas:
        return obj, ""
    cmd = [nvcc(), "-c", str(src), "-o", str(obj)] + _flags(ptxas)
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, ptxas=False):
    OBJ.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    srcs = sorted(SRC.glob("*.cu"))
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas, verbose), srcs))
    objs = [o for o, _ in results]
    if ptxas:
        for _, log in results:
            sys.stdout.write(log)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), "-shared", "-o", str(LIB)] + [str(o) for o in objs] + ARCH + [
            "-ccbin", host_compiler(), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v resource usage")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas))
