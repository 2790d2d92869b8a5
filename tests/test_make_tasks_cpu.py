"""The row samplers' work split (make_tasks, macau_b200/csrc/host_util.h), compiled with g++ and
checked on the CPU at every split threshold the autotuner may pick: coverage, alignment, part
lengths, split counters and slots, and the stable descending order."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CUDA = Path("/usr/local/cuda")


@pytest.mark.skipif(shutil.which("g++") is None or not (CUDA / "include").exists(),
                    reason="needs g++ and the CUDA headers")
def test_make_tasks_invariants(tmp_path):
    exe = tmp_path / "make_tasks_check"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'macau_b200' / 'csrc'}",
                    f"-I{CUDA / 'include'}", str(ROOT / "tests" / "cpp" / "make_tasks_check.cpp"),
                    "-o", str(exe), f"-L{CUDA / 'lib64'}", "-lcudart",
                    f"-Wl,-rpath,{CUDA / 'lib64'}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "OK", (r.stdout, r.stderr)
