"""Extracts the known-answer fixtures of the reference's C++ unit tests into JSON.

The reference (jaak-s/macau 0.5.3) cannot be compiled in this environment (Eigen 3.3.7 is
downloaded at build time and the libfastsparse submodule is empty), so its own golden values
are read as *text* from ``lib/macau-cpp/tests.cpp`` and stored as small fixtures.  The tests
read only the JSON this script writes (``reference_tests_cpp.json``); the reference tree is
needed only to regenerate it:

    python tests/golden/extract_reference_fixtures.py <path of the reference checkout>

Eigen comma initialisers (``M << a, b, ...;``) fill matrices row by row; the JSON keeps that
row-major order together with the matrix shape declared in the test.
"""
import ast
import json
import operator
import re
import sys
from pathlib import Path

CASES = [
    "linop/A_mul_Bx(csr)",
    "linop/AtA_mul_Bx(csr)",
    "SparseFeat/compute_uhat",
    "SparseFeat/solve_blockcg",
    "SparseFeat/solve_blockcg_1_0",
    "MatrixXd/compute_uhat",
    "linop/solve_blockcg_dense",
    "latentprior/sample_lambda_beta",
    "bpmfutils/eval_rmse",
]

_OPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul,
        ast.Div: operator.truediv, ast.USub: operator.neg, ast.UAdd: operator.pos}


def _num(expr):
    """Evaluates a numeric literal expression such as ``(3.0 + 4.0) / 2``."""
    def ev(node):
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
            return node.value
        if isinstance(node, ast.BinOp) and type(node.op) in _OPS:
            return _OPS[type(node.op)](ev(node.left), ev(node.right))
        if isinstance(node, ast.UnaryOp) and type(node.op) in _OPS:
            return _OPS[type(node.op)](ev(node.operand))
        raise ValueError(expr)
    return float(ev(ast.parse(expr.strip(), mode="eval").body))


def _case_bodies(src):
    out = {}
    heads = list(re.finditer(r'TEST_CASE\(\s*"([^"]+)"', src))
    for k, m in enumerate(heads):
        end = heads[k + 1].start() if k + 1 < len(heads) else len(src)
        out[m.group(1)] = (src[m.start():end], src[:m.start()].count("\n") + 1)
    return out


def _parse(body):
    """Returns the ordered statements of one TEST_CASE body."""
    shapes = {}
    for m in re.finditer(r"Eigen::(?:MatrixXd|SparseMatrix<double>)\s+([^;]+);", body):
        for d in re.finditer(r"(\w+)\((\d+),\s*(\d+)\)", m.group(1)):
            shapes[d.group(1)] = [int(d.group(2)), int(d.group(3))]
    for d in re.finditer(r"(\w+)\.resize\((\d+),\s*(\d+)\)", body):
        shapes[d.group(1)] = [int(d.group(2)), int(d.group(3))]
    stmts = []
    pat = re.compile(
        r"(?P<arr>(?:int|double)\s+(?P<an>\w+)\[\d+\]\s*=\s*\{(?P<av>[^}]*)\}\s*;)"
        r"|(?P<init>\b(?P<mn>\w+)\s*<<(?P<mv>[^;]*);)"
        r"|(?P<scal>\bdouble\s+(?P<sn>\w+)\s*=\s*(?P<sv>[-+0-9.eE]+)\s*;)"
        r"|(?P<req>REQUIRE\s*\((?P<rq>.*?)\)\s*;[ \t]*(?://[^\n]*)?$)"
        r"|(?P<call>\b(?P<cn>eval_rmse|posterior_lambda_beta|solve_blockcg)\s*\((?P<ca>[^;]*)\)\s*;)",
        re.M)
    for m in pat.finditer(body):
        if m.group("arr"):
            vals = [v for v in re.split(r"[,\s]+", m.group("av").strip()) if v]
            stmts.append({"kind": "array", "name": m.group("an"), "values": [_num(v) for v in vals]})
        elif m.group("init"):
            vals = [v for v in m.group("mv").replace("\n", " ").split(",") if v.strip()]
            stmts.append({"kind": "matrix", "name": m.group("mn"),
                          "shape": shapes.get(m.group("mn")), "values": [_num(v) for v in vals]})
        elif m.group("scal"):
            stmts.append({"kind": "scalar", "name": m.group("sn"), "value": _num(m.group("sv"))})
        elif m.group("req"):
            stmts.append({"kind": "require", "text": " ".join(m.group("rq").split())})
        elif m.group("call"):
            stmts.append({"kind": "call", "fn": m.group("cn"),
                          "args": [a.strip() for a in m.group("ca").split(",")]})
    return stmts


def _require_value(text):
    """'pred(0) == Approx((3.0 + 4.0) / 2)' -> ('pred(0)', 3.5, True)."""
    m = re.match(r"(.+?)\s*(==|<=|>=|<|>)\s*(Approx\((.*)\)|(.*))$", text)
    lhs, op = m.group(1).strip(), m.group(2)
    rhs = m.group(4) if m.group(4) is not None else m.group(5)
    try:
        val = _num(rhs)
    except ValueError:
        return {"lhs": lhs, "op": op, "rhs": rhs.strip(), "approx": m.group(4) is not None}
    return {"lhs": lhs, "op": op, "value": val, "approx": m.group(4) is not None}


def main(ref_root):
    path = Path(ref_root) / "lib" / "macau-cpp" / "tests.cpp"
    src = path.read_text()
    bodies = _case_bodies(src)
    out = {"source": "lib/macau-cpp/tests.cpp (jaak-s/macau 0.5.3)", "cases": {}}
    for name in CASES:
        body, line = bodies[name]
        stmts = _parse(body)
        for s in stmts:
            if s["kind"] == "require":
                s.update(_require_value(s["text"]))
        out["cases"][name] = {"line": line, "statements": stmts}
    dst = Path(__file__).with_name("reference_tests_cpp.json")
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {dst} ({len(out['cases'])} cases)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract_reference_fixtures.py <path of the reference checkout>")
    main(sys.argv[1])
