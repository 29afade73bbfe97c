"""Host-side checks of the C ABI that need no GPU: the library loads, exports
every symbol the headers declare, validates arguments, and reports "no device"
as the try_create contract asks (src/solvers/cuda_direct_solver.cpp:140-164)."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import orrery_b200 as ob
from orrery_b200 import initial_conditions as ic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for match in re.finditer(r"\b(ob_[a-z0-9_]+)\s*\(", text):
            names.add(match.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(ob.library_path()):
        from orrery_b200 import build
        build.build()
    return ob.load_library()


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_text(lib):
    assert "sm_100a" in ob.version()
    assert isinstance(lib.ob_last_error(), bytes)


def test_invalid_parameters_are_rejected_before_the_device(lib):
    handle = C.c_void_p()
    bad = ob.make_params(kind=7)
    assert lib.ob_solver_create(C.byref(bad), C.byref(handle)) == ob.ERROR_INVALID_ARGUMENT
    assert handle.value is None
    bad = ob.make_params()
    bad.softening_squared = -1.0
    assert lib.ob_solver_create(C.byref(bad), C.byref(handle)) == ob.ERROR_INVALID_ARGUMENT
    bad.softening_squared = float("nan")
    assert lib.ob_solver_create(C.byref(bad), C.byref(handle)) == ob.ERROR_INVALID_ARGUMENT
    bad = ob.make_params(kind=ob.SOLVER_TREE, precision="split")
    assert lib.ob_solver_create(C.byref(bad), C.byref(handle)) == ob.ERROR_UNSUPPORTED
    assert lib.ob_solver_create(None, C.byref(handle)) == ob.ERROR_INVALID_ARGUMENT


def test_null_handles_are_errors_not_crashes(lib):
    counts = ob.Counts()
    assert lib.ob_solver_counts(None, C.byref(counts)) == ob.ERROR_INVALID_ARGUMENT
    assert lib.ob_system_step(None, 0, 1e-3, 1) == ob.ERROR_INVALID_ARGUMENT
    lib.ob_solver_destroy(None)
    lib.ob_system_destroy(None)


def test_negative_counts_are_refused_not_wrapped(lib):
    # A uint64_t cannot hold -1; passed through, it would become 2^64 - 1
    # steps. The binding's argument type refuses it (ctypes reports that as an
    # ArgumentError), and the Python surface refuses it first with an
    # invalid-argument error, before anything reaches the library.
    with pytest.raises(C.ArgumentError):
        lib.ob_system_step(None, 0, 1e-3, -1)
    with pytest.raises(C.ArgumentError):
        lib.ob_system_step(None, 0, 1e-3, 1 << 64)
    assert lib.ob_system_step(None, 0, 1e-3, np.uint64(3)) == ob.ERROR_INVALID_ARGUMENT
    system = ob.DeviceSystem.__new__(ob.DeviceSystem)  # no device: refused before the call
    system._lib, system._handle = lib, None
    for call in (lambda: system.step(1e-3, -1), lambda: system.step_async(1e-3, -2),
                 lambda: system.write_checkpoint("never.ck", -1),
                 lambda: ob.work_units(1000, -1, "direct")):
        with pytest.raises(ob.OrreryError, match="must be in") as e:
            call()
        assert e.value.code == ob.ERROR_INVALID_ARGUMENT
    with pytest.raises(TypeError):
        ob.work_units(1000, 2.5, "direct")  # a count is an integer, as the reference's Index is


def test_try_create_without_a_device_returns_none(lib):
    if ob.device_count() > 0:
        pytest.skip("a device is present; the no-device contract is tested without one")
    assert ob.B200DirectSolver.try_create(0.01) is None
    assert ob.B200TreeSolver.try_create(0.01) is None
    handle = C.c_void_p()
    params = ob.make_params()
    assert lib.ob_system_create(C.byref(params), 16, C.byref(handle)) == ob.ERROR_NO_DEVICE


def test_plummer_generator_is_seeded_and_centred():
    a = ic.plummer_sphere(3000, seed=7)
    b = ic.plummer_sphere(3000, seed=7)
    c = ic.plummer_sphere(3000, seed=8)
    assert np.array_equal(a["x"], b["x"]) and not np.array_equal(a["x"], c["x"])
    assert abs(a["m"].sum() - 1.0) < 1e-12
    com = np.array([(a[k] * a["m"]).sum() for k in ("x", "y", "z")])
    assert np.all(np.abs(com) < 1e-12)
    # Half-mass radius of a Plummer sphere: a / sqrt(2^{2/3} - 1) ~ 1.305 a.
    r = np.sqrt(a["x"] ** 2 + a["y"] ** 2 + a["z"] ** 2)
    assert 1.15 < np.median(r) < 1.45


def test_collision_generator_geometry():
    g = ic.galaxy_collision(20000, seed=3)
    assert len(g["x"]) == 20000
    assert abs(g["m"].sum() - 1.0) < 1e-12
    assert np.allclose(g["m"], g["m"][0])
    b = ic.collision_impact_parameter(1.0, 20.0, 0.8, 3.0)
    assert 0 < b < 20


def test_positions_are_accepted_in_every_documented_layout():
    # ForceSolver::evaluate takes three spans; the Python surface accepts
    # three arrays, (N, 3) or (3, N), and refuses anything else.
    rng = np.random.default_rng(3)
    xyz = [rng.normal(size=5) for _ in range(3)]
    for positions in (tuple(xyz), list(xyz), np.stack(xyz, axis=1), np.stack(xyz, axis=0)):
        got = ob._split_xyz(positions)
        assert all(np.array_equal(g, w) for g, w in zip(got, xyz))
        assert all(g.dtype == np.float64 and g.flags.c_contiguous for g in got)
    square = rng.normal(size=(3, 3))  # ambiguous: read as (N, 3), rows are particles
    assert all(np.array_equal(g, square[:, k]) for k, g in enumerate(ob._split_xyz(square)))
    with pytest.raises(ValueError):
        ob._split_xyz(np.zeros((4, 4)))
    with pytest.raises(ValueError):
        ob._split_xyz(np.zeros(6))


def test_noalloc_ordering_checks_its_arguments_before_the_device(lib):
    # Refusals come before any CUDA call, so they hold on a machine without a
    # device too: above the fixed scratch's capacity, and NULL arrays.
    fn = lib.ob_morton_order_noalloc
    fn.argtypes = [C.c_uint64] + [C.c_void_p] * 7
    fn.restype = C.c_int
    assert fn((1 << 20) + 1, None, None, None, None, None, None, None) == ob.ERROR_CAPACITY
    assert b"1048576" in lib.ob_last_error()
    fake = C.c_void_p(16)  # never dereferenced: the NULL check refuses first
    assert fn(10, fake, fake, None, fake, fake, None, None) == ob.ERROR_INVALID_ARGUMENT
