"""The code in INTEGRATION.md is what the package and the reference provide.

The C++ listings (a run through the adapters, a run with output) are compiled
here with g++ -fsyntax-only against the reference's include tree, the
adapter header and this library's C header, so that a change on either side
that breaks them shows up; the reference checkout comes from
ORRERY_REFERENCE_ROOT or the one build() used, and the compile is skipped
where there is none. The Python listings are parsed and their ob.* calls
checked against the package.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def listings():
    with open(os.path.join(ROOT, "INTEGRATION.md")) as fh:
        return re.findall(r"```cpp\n(.*?)```", fh.read(), re.S)


def test_there_are_listings():
    assert len(listings()) >= 2


def python_listings():
    with open(os.path.join(ROOT, "INTEGRATION.md")) as fh:
        return re.findall(r"```python\n(.*?)```", fh.read(), re.S)


@pytest.mark.parametrize("index", range(len(python_listings())))
def test_python_listing_parses_and_calls_what_the_package_has(index):
    # Each `ob.<name>(...)` call names something the package exports and
    # passes only keywords its signature accepts.
    import ast
    import inspect

    import orrery_b200 as ob

    tree = ast.parse(python_listings()[index])
    for node in ast.walk(tree):
        if not (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute) and
                isinstance(node.func.value, ast.Name) and node.func.value.id == "ob"):
            continue
        target = getattr(ob, node.func.attr, None)
        assert target is not None, f"ob.{node.func.attr} does not exist"
        params = inspect.signature(target).parameters
        if any(p.kind is p.VAR_KEYWORD for p in params.values()):
            continue
        for kw in node.keywords:
            if kw.arg is not None:
                assert kw.arg in params, f"ob.{node.func.attr} takes no {kw.arg}="


@pytest.mark.parametrize("index", range(len(listings())))
def test_listing_compiles_against_the_reference(tmp_path, index):
    import oracle

    root = oracle.reference_root()
    if shutil.which("g++") is None or root is None:
        pytest.skip("g++ or the reference checkout is not available here "
                    "(set ORRERY_REFERENCE_ROOT to the reference's checkout)")
    source = tmp_path / f"listing{index}.cpp"
    source.write_text(listings()[index])
    out = subprocess.run(["g++", "-std=c++20", "-fsyntax-only",
                          f"-I{os.path.join(root, 'include')}",
                          f"-I{os.path.join(ROOT, 'orrery_b200', 'adapter')}",
                          f"-I{os.path.join(ROOT, 'include')}", str(source)],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-3000:]
