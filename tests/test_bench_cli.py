"""bench.py imports without a device, parses its defaults, and defines every
leg its runner calls (a leg that went missing would otherwise only fail on a GPU)."""
import ast
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_defines_every_function_it_calls():
    src = open(os.path.join(ROOT, "bench.py")).read()
    tree = ast.parse(src)
    defined = {n.name for n in tree.body if isinstance(n, (ast.FunctionDef, ast.ClassDef))}
    called = {n.func.id for n in ast.walk(tree)
              if isinstance(n, ast.Call) and isinstance(n.func, ast.Name)}
    builtins = set(dir(__builtins__)) if isinstance(__builtins__, dict) is False else set(__builtins__)
    imported = set()
    for n in ast.walk(tree):
        if isinstance(n, (ast.Import, ast.ImportFrom)):
            imported |= {(a.asname or a.name).split(".")[0] for a in n.names}
    missing = sorted(c for c in called - defined - imported - builtins
                     if c not in {"print", "len", "sum", "max", "min", "sorted", "range", "float",
                                  "int", "str", "open", "zip", "enumerate", "round", "isinstance",
                                  "dict", "list", "set", "abs", "any", "all", "getattr"})
    assert not missing, missing


def test_bench_parses_defaults(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert (a.gpus, a.impl, a.size, a.ensemble, a.serve_requests) == (1, "ours", 8192, 256, 32)
    assert a.warmup >= 3
    for f in ("run_ours", "run_reference", "run_ensemble", "run_serving", "time_fused",
              "time_e2e", "time_batch_copies", "cpu_reference"):
        assert callable(getattr(bench, f))
    d = bench.describe(8192)
    assert d["cells"] == 8192 * 8192 and "workload" in d
