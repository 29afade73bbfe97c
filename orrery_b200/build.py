"""Builds the sm_100a CUDA library ``_lib/liborrery_b200.so`` in-tree.

Every translation unit under ``csrc/`` is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared library
exposing the C ABI declared in ``include/orrery_b200.h``. ``python -m
orrery_b200.build`` runs it; ``__graft_entry__.build()`` calls :func:`build`.
"""
from __future__ import annotations

import concurrent.futures as futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(OUT, "obj")
LIBRARY = os.path.join(OUT, "liborrery_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]

# Per-file flags. Files that restate the reference's FP64 arithmetic bit for
# bit are compiled without multiply-add contraction; they also use explicitly
# rounded intrinsics, so this is belt and braces.
EXTRA = {
    "direct.cu": ["-ftz=true"],
    "integrate.cu": ["--fmad=false"],
    "tree.cu": ["--fmad=false"],
    "walk.cu": ["-ftz=true"],
    "walk_f64.cu": ["--fmad=false"],
}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(source: str) -> tuple[str, str]:
    src = os.path.join(CSRC, source)
    obj = os.path.join(OBJ, source.replace(".cu", ".o"))
    cmd = [nvcc(), *ARCH, *COMMON, *EXTRA.get(source, []), "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def _stale(objects) -> bool:
    if not os.path.exists(LIBRARY):
        return True
    lib_time = os.path.getmtime(LIBRARY)
    inputs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inputs += [os.path.join(ROOT, "include", "orrery_b200.h"), __file__]
    return any(os.path.getmtime(p) > lib_time for p in inputs)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the library if any source is newer than it; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    sources = _sources()
    if not force and not _stale(sources):
        return LIBRARY
    logs = []
    with futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as pool:
        for obj, log in pool.map(_compile, sources):
            logs.append((obj, log))
    with open(os.path.join(OUT, "ptxas.log"), "w") as fh:
        for obj, log in logs:
            fh.write(f"== {os.path.basename(obj)}\n{log}\n")
    objects = [o for o, _ in logs]
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIBRARY, *objects, "-lcuda"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        for obj, log in logs:
            print(f"== {os.path.basename(obj)}\n{log}")
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
