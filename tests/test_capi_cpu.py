"""CPU-side checks of the drop-in boundary: the C-ABI library loads, exports every entry point
declared in include/*.h, reports a missing GPU with its own error code, and the Python mirror of
macau.pyx validates arguments like the reference (no GPU needed for any of this)."""
import re
from pathlib import Path

import numpy as np
import pandas as pd
import pytest
import scipy.sparse as sp

import macau_b200
from macau_b200 import _lib, build

ROOT = Path(__file__).resolve().parents[1]


def declared_entry_points():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+[\s\*]+(mg_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not _lib.LIB_PATH.exists():
        build.build()
    return _lib.lib()


def test_library_exports_every_declared_symbol(lib):
    names = declared_entry_points()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.EXPORTED, n


def test_create_without_gpu_reports_error(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(_lib.MacauError) as e:
        _lib.Sampler(8, 1.0)
    assert e.value.code in (-7, -4)


def test_python_api_validation_errors():
    Y = sp.random(10, 20, density=0.2, format="coo", random_state=0)
    with pytest.raises(ValueError):  # test_macau.py:159-162 (side list too long)
        macau_b200.macau(Y, verbose=False, side=[None, None, None])
    with pytest.raises(ValueError):
        macau_b200.macau(Y, verbose=False, side="x")
    with pytest.raises(ValueError):
        macau_b200.macau(Y, verbose=False, precision="probit")
    with pytest.raises(ValueError):  # make_one_prior takes sparse side information only
        macau_b200.macau(Y, verbose=False, univariate=True, side=[np.zeros((10, 2)), None])
    with pytest.raises(TypeError):
        macau_b200.macau(np.zeros((3, 3)), verbose=False)
    with pytest.raises(ValueError):
        macau_b200.macau(Y, Ytest=sp.random(5, 5, density=0.2, format="coo"), verbose=False)
    with pytest.raises(ValueError):
        macau_b200.macau(Y, verbose=False, compute="fp16")
    with pytest.raises(ValueError):
        macau_b200.blockcg(Y, np.zeros((2, 20)), 0.5)  # B must be order='F'


def test_make_train_test():  # test_macau.py:174-179
    X = sp.random(15, 10, density=0.2, format="coo", random_state=1)
    Xtr, Xte = macau_b200.make_train_test(X, 0.5)
    assert X.nnz == Xtr.nnz + Xte.nnz
    assert np.linalg.norm((X - Xtr - Xte).toarray()) == 0.0


def test_make_train_test_df():  # test_macau.py:181-196
    import itertools
    idx = list(itertools.product(np.arange(10), np.arange(8), np.arange(3)))
    df = pd.DataFrame(np.asarray(idx), columns=["A", "B", "C"])
    df["value"] = np.arange(10.0 * 8.0 * 3.0)
    Ytr, Yte = macau_b200.make_train_test_df(df, 0.4)
    assert Ytr.shape[0] == df.shape[0] * 0.6
    assert Yte.shape[0] == df.shape[0] * 0.4


def test_dataframe_tensor_is_rejected():
    df = pd.DataFrame({"A": [0, 1], "B": [0, 1], "C": [0, 0], "value": [1.0, 2.0]})
    with pytest.raises(ValueError, match="Tensor"):
        macau_b200.macau(df, verbose=False)


def test_workload_generators_shapes():
    from macau_b200 import workloads
    w = workloads.bpmf_powerlaw(scale=0.01)
    assert len(w["vals"]) > 0 and w["vals"].min() >= 0.5 and w["vals"].max() <= 5.0
    assert np.all((w["vals"] * 2) == np.round(w["vals"] * 2))
    w = workloads.macau_side(scale=0.01)
    fr, fc, fv, shp = w["side"]
    assert fv is None and fc.max() < shp[1]


def test_ctrl_c_stops_after_the_current_iteration(capsys):
    # macau()'s sweep loop runs inside _StopOnInterrupt: SIGINT sets a flag and prints the
    # reference's note (macau.cpp:30-35) instead of raising, and the previous handler comes back
    import os
    import signal
    import time

    from macau_b200.macau import _StopOnInterrupt

    before = signal.getsignal(signal.SIGINT)
    with _StopOnInterrupt() as stop:
        assert not stop.requested
        os.kill(os.getpid(), signal.SIGINT)
        for _ in range(100):
            if stop.requested:
                break
            time.sleep(0.01)
        assert stop.requested
    assert signal.getsignal(signal.SIGINT) is before
    assert _StopOnInterrupt.MESSAGE in capsys.readouterr().out


def test_cpp_host_class_builds_and_reports_errors(tmp_path):
    # include/macau_b200.hpp compiles against the header, links the library, and turns the
    # library's error into std::runtime_error (here: no GPU in this process's view)
    import shutil

    from macau_b200 import workloads
    from tests import cpp_host

    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present (the GPU run is compared with the ctypes path elsewhere)")
    exe = cpp_host.build(tmp_path)
    w = workloads.bpmf_uniform(nrow=50, ncol=40, nobs=600, seed=1)
    cpp_host.write_data(tmp_path / "d.bin", w, 4, 2, 2)
    code, out, err = cpp_host.run(exe, tmp_path / "d.bin", 5)
    assert code == 2 and out.get("ERROR"), (code, out, err)
    assert "CUDA" in out["ERROR"] or "GPU" in out["ERROR"] or "device" in out["ERROR"], out
