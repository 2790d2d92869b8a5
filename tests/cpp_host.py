"""Builds and runs tests/cpp/macau_cpp_host.cpp, the C++ host over include/macau_b200.hpp."""
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
CUDA_LIB = "/usr/local/cuda/lib64"


def build(tmp_path):
    exe = tmp_path / "macau_cpp_host"
    lib_dir = ROOT / "macau_b200" / "_lib"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "cpp" / "macau_cpp_host.cpp"), "-o", str(exe),
                    f"-L{lib_dir}", "-lmacau_b200", f"-Wl,-rpath,{lib_dir}",
                    f"-Wl,-rpath,{CUDA_LIB}", f"-Wl,-rpath-link,{CUDA_LIB}"], check=True)
    return exe


def write_data(path, w, K, burnin, nsamples):
    n, t = len(w["vals"]), len(w["tvals"])
    with open(path, "wb") as f:
        np.array([w["shape"][0], w["shape"][1], n, t, K, burnin, nsamples], np.int32).tofile(f)
        np.asarray(w["rows"], np.int32).tofile(f)
        np.asarray(w["cols"], np.int32).tofile(f)
        np.asarray(w["vals"], np.float64).tofile(f)
        np.asarray(w["trows"], np.int32).tofile(f)
        np.asarray(w["tcols"], np.int32).tofile(f)
        np.asarray(w["tvals"], np.float64).tofile(f)


def run(exe, data, seed):
    r = subprocess.run([str(exe), str(data), str(seed)], capture_output=True, text=True,
                       timeout=300)
    out = {}
    for line in r.stdout.splitlines():
        k, _, v = line.partition(" ")
        out[k] = v
    return r.returncode, out, r.stderr
