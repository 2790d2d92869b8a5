"""Pins the CPU oracle to the reference's own known-answer tests (lib/macau-cpp/tests.cpp),
read from the committed fixture tests/golden/reference_tests_cpp.json, and to the published
Philox-4x32-10 known-answer vectors."""
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as orc

FIX = json.loads((Path(__file__).parent / "golden" / "reference_tests_cpp.json").read_text())


def approx(a, b):
    """Catch v1 Approx: |a-b| < 100*FLT_EPSILON*(1 + max(|a|,|b|))."""
    return abs(a - b) < 100 * np.finfo(np.float32).eps * (1.0 + max(abs(a), abs(b)))


def case(name):
    """Returns ({name: value}, [statements]) for a tests.cpp TEST_CASE; matrices row-major."""
    st = FIX["cases"][name]["statements"]
    env = {}
    for s in st:
        if s["kind"] == "array":
            env[s["name"]] = np.array(s["values"])
        elif s["kind"] == "matrix" and s["name"] not in env:
            env[s["name"]] = np.array(s["values"]).reshape(s["shape"])
        elif s["kind"] == "scalar":
            env[s["name"]] = s["value"]
    return env, st


def fixture_F(env, nrow=6, ncol=4, with_vals=True, binary=None):
    """The 6x4 fixture matrix of tests.cpp:17-18; binary => no value array (SparseFeat)."""
    vals = env["vals"] if with_vals else np.ones(len(env["rows"]))
    m = sp.coo_matrix((vals, (env["rows"].astype(int), env["cols"].astype(int))),
                      shape=(nrow, ncol))
    binary = (not with_vals) if binary is None else binary
    return orc.Csr.from_scipy(m, binary), orc.Csr.from_scipy(m.T, binary)


def test_philox_known_answers():
    # Published Philox-4x32-10 known-answer vectors (Random123 kat_vectors).
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in kat:
        assert tuple(int(x) for x in orc.philox(ctr, key)) == want


def test_a_mul_bx_csr():  # tests.cpp:66-78
    env, _ = case("linop/A_mul_Bx(csr)")
    F, _ = fixture_F(env)
    X = orc.csr_mul_bn(F, env["B"].T)  # (6, 2) == X^T
    assert np.linalg.norm(X - env["Xtr"].T) == pytest.approx(0, abs=1e-12)


def test_ata_mul_bx_csr():  # tests.cpp:80-100
    env, _ = case("linop/AtA_mul_Bx(csr)")
    F, Ft = fixture_F(env)
    out = orc.ata_mul_bx(F, Ft, env["reg"], env["B"].T)
    Xd = env["X"]
    want = (Xd.T @ Xd @ env["B"].T + env["reg"] * env["B"].T)
    assert np.linalg.norm(out - want) < 1e-12


def test_compute_uhat_binary():  # tests.cpp:102-121
    env, _ = case("SparseFeat/compute_uhat")
    F, _ = fixture_F(env, with_vals=False)
    uhat = orc.csr_mul_bn(F, env["beta"].T)  # (6, 3)
    for i in range(3):
        for j in range(6):
            assert approx(uhat[j, i], env["uhat_true"][i, j])


def test_compute_uhat_dense_as_csr():  # tests.cpp:163-181 (dense features through CSR values)
    env, _ = case("MatrixXd/compute_uhat")
    F = orc.Csr.from_scipy(sp.csr_matrix(env["feat"]))
    uhat = orc.csr_mul_bn(F, env["beta"].T)
    for i in range(2):
        for j in range(6):
            assert approx(uhat[j, i], env["uhat_true"][i, j])


def test_blockcg_one_rhs():  # tests.cpp:123-138
    env, st = case("SparseFeat/solve_blockcg")
    F, Ft = fixture_F(env, with_vals=False)
    X, niter = orc.blockcg(F, Ft, 0.5, env["B"].T, 1e-6)
    for j in range(4):
        assert approx(X[j, 0], env["X_true"][0, j])
    limit = [s for s in st if s["kind"] == "require" and s["lhs"] == "niter"][0]["value"]
    assert niter <= limit


@pytest.mark.parametrize("name,blocked", [("SparseFeat/solve_blockcg_1_0", True),
                                          ("linop/solve_blockcg_dense", False)])
def test_blockcg_three_rhs(name, blocked):  # tests.cpp:141-161, 183-207
    env, _ = case(name)
    # SparseFeat => binary CSR; the dense 0/1 matrix => CSR with explicit 1.0 values.
    F, Ft = fixture_F(env, with_vals=False, binary=name.startswith("SparseFeat"))
    if blocked:
        X, _ = orc.blockcg(F, Ft, 0.5, env["B"].T, 1e-6, blocksize=1, excess=0)
    else:
        X, _ = orc.blockcg(F, Ft, 0.5, env["B"].T, 1e-6)
    for i in range(3):
        for j in range(4):
            assert approx(X[j, i], env["X_true"][i, j])


def test_posterior_lambda_beta():  # tests.cpp:241-254
    env, st = case("latentprior/sample_lambda_beta")
    call = [s for s in st if s["kind"] == "call"][0]
    nu, mu = float(call["args"][2]), float(call["args"][3])
    b, c = orc.posterior_lambda_beta(env["beta"].T, env["Lambda_u"], nu, mu)
    want = {s["lhs"]: s["value"] for s in st if s["kind"] == "require" and "value" in s}
    assert approx(b, want["post.first"])
    assert approx(c, want["post.second"])
    assert orc.gamma(1234, 0, "lambda_beta", 0, 0, b) * c > 0


def test_eval_rmse_sequence():  # tests.cpp:552-591
    env, st = case("bpmfutils/eval_rmse")
    pred = np.zeros(1)
    var = np.zeros(1)
    U = V = None
    results = {}
    step = 0
    for s in st:
        if s["kind"] == "matrix":
            if s["name"] == "U":
                U = np.array(s["values"]).reshape(1, 2)  # one column of K=2
            else:
                V = np.array(s["values"]).reshape(1, 2)
        elif s["kind"] == "call":
            n = int(s["args"][1])
            r1, ravg = orc.eval_rmse([0], [0], [4.5], n, pred, var, V, U, env["mean_value"])
            results = {"pred(0)": pred[0], "pred_var(0)": var[0],
                       f"rmse{step}.first": r1, f"rmse{step}.second": ravg}
            step += 1
        elif s["kind"] == "require":
            got = results[s["lhs"]]
            if s["approx"]:
                assert approx(got, s["value"]), s["text"]
            else:
                assert got == s["value"], s["text"]
    assert step == 3
