"""The product path never routes through the oracle: nothing in the package
(Python mirror, CUDA and C++ sources, build recipe) names it, and bench.py
imports it only in the functions of the CPU baseline.  Static checks
over the sources; no GPU."""
import ast
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rustfs-erasure-codec_b200")


def test_package_never_names_the_oracle():
    hits = []
    for dirpath, _, files in os.walk(PKG):
        if "_build" in dirpath:
            continue
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".hpp", ".h", ".txt")):
                path = os.path.join(dirpath, f)
                with open(path, errors="replace") as fh:
                    if re.search(r"\boracle\b", fh.read()):
                        hits.append(os.path.relpath(path, ROOT))
    assert hits == []


def test_bench_imports_the_oracle_only_for_the_cpu_baseline():
    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    owners = set()
    for fn in ast.walk(tree):
        if isinstance(fn, (ast.FunctionDef, ast.AsyncFunctionDef)):
            for node in ast.walk(fn):
                if isinstance(node, ast.Import) and any(a.name == "oracle" for a in node.names):
                    owners.add(fn.name)
                if isinstance(node, ast.ImportFrom) and node.module == "oracle":
                    owners.add(fn.name)
    top = [n for n in tree.body if isinstance(n, (ast.Import, ast.ImportFrom))
           and ("oracle" in [a.name for a in getattr(n, "names", [])] or getattr(n, "module", None) == "oracle")]
    # cpu_sample times the CPU baseline; cpu_widths asks it which vector
    # widths this host's baseline can run.
    assert top == [] and owners == {"cpu_sample", "cpu_widths"}
