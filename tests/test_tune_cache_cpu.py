"""The autotuner's keys and choice cache (macau_b200/csrc/tune.h), compiled with g++ and run on
the CPU: one process writes choices to the file cache, a second reads them back."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_tune_key_and_file_cache(tmp_path):
    exe = tmp_path / "tune_cache_check"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'macau_b200' / 'csrc'}",
                    str(ROOT / "tests" / "cpp" / "tune_cache_check.cpp"), "-o", str(exe)],
                   check=True)
    cache = tmp_path / "tune.txt"
    for step in ("write", "read"):
        r = subprocess.run([str(exe), step, str(cache)], capture_output=True, text=True)
        assert r.returncode == 0 and r.stdout.strip() == "OK", (step, r.stdout, r.stderr)
    assert len(cache.read_text().splitlines()) == 2
