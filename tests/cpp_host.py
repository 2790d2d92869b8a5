"""Builds and runs the C++ hosts of tests/cpp: macau_cpp_host.cpp (the host class of
include/macau_b200.hpp) and prior_adapter_check.cpp (the adapters of
include/macau_b200_priors.hpp behind the reference's ILatentPrior / Macau interfaces)."""
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
CUDA_LIB = "/usr/local/cuda/lib64"


def build(tmp_path, name="macau_cpp_host"):
    exe = tmp_path / name
    lib_dir = ROOT / "macau_b200" / "_lib"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    f"-I{ROOT / 'include'}", f"-I{ROOT / 'tests' / 'cpp'}",
                    str(ROOT / "tests" / "cpp" / f"{name}.cpp"), "-o", str(exe),
                    f"-L{lib_dir}", "-lmacau_b200", f"-Wl,-rpath,{lib_dir}",
                    f"-Wl,-rpath,{CUDA_LIB}", f"-Wl,-rpath-link,{CUDA_LIB}"], check=True)
    return exe


def write_data(path, w, K, burnin, nsamples, side=None):
    """side: None, or (rows, cols, nfeat) of a binary mode-0 side matrix, appended after the
    test set for prior_adapter_check (macau_cpp_host ignores what follows the test set)."""
    n, t = len(w["vals"]), len(w["tvals"])
    with open(path, "wb") as f:
        np.array([w["shape"][0], w["shape"][1], n, t, K, burnin, nsamples], np.int32).tofile(f)
        np.asarray(w["rows"], np.int32).tofile(f)
        np.asarray(w["cols"], np.int32).tofile(f)
        np.asarray(w["vals"], np.float64).tofile(f)
        np.asarray(w["trows"], np.int32).tofile(f)
        np.asarray(w["tcols"], np.int32).tofile(f)
        np.asarray(w["tvals"], np.float64).tofile(f)
        if side is None:
            np.array([0, 0], np.int32).tofile(f)
        else:
            fr, fc, nfeat = side
            np.array([len(fr), nfeat], np.int32).tofile(f)
            np.asarray(fr, np.int32).tofile(f)
            np.asarray(fc, np.int32).tofile(f)


def run(exe, data, seed):
    r = subprocess.run([str(exe), str(data), str(seed)], capture_output=True, text=True,
                       timeout=300)
    out = {}
    for line in r.stdout.splitlines():
        k, _, v = line.partition(" ")
        out[k] = v
    return r.returncode, out, r.stderr
