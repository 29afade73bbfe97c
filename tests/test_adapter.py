"""The C++ adapters (orrery_b200/adapter/b200_solver.hpp) under the reference's
own integrators.

B200DirectSolver and B200TreeSolver are orrery::solvers::ForceSolver
implementations; B200Integrator is an orrery::integrators::Integrator that
steps on the device. oracle/ref_adapter_shim.cpp, compiled against the
reference's headers and linked with the reference's own sources and this
library, hands them to the reference's VelocityVerlet, Yoshida4 and
RungeKutta4 (src/integrators/velocity_verlet.cpp:59-72, yoshida4.cpp:45-59,
runge_kutta4.cpp:64-139) exactly as sim::Simulation would. In FP64 every
trajectory must equal, bit for bit, the same integrator's run over the
reference's DirectSolver / BarnesHutSolver (scalar kernels); in FP32 and the
split form, the forces stay within the bounds the other GPU tests state.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle

from conftest import relative_errors

KEYS = oracle.AdapterDriver.STATE


@pytest.fixture(scope="module")
def driver():
    if not oracle.AdapterDriver.built():
        pytest.skip("the adapter driver (oracle/_ref/libref_adapter.so) is not built here; "
                    "build() builds it where ORRERY_REFERENCE_ROOT names the reference")
    return oracle.AdapterDriver()


@pytest.fixture(scope="module")
def plummer(reference):
    # The reference's own sampler, so both sides start from its bits.
    return reference.plummer(2048, seed=20260903)


def _state(p, n=None):
    n = n or len(p["m"])
    return {k: p[k][:n] for k in ("x", "y", "z", "vx", "vy", "vz")}, p["m"][:n]


# ---------------------------------------------------------------- host (CPU)

@pytest.mark.parametrize("method", ["vv", "yoshida4", "rk4"])
def test_integrator_traits_are_the_reference_integrators(driver, method):
    assert driver.traits(True, method) == driver.traits(False, method)


def test_try_create_gives_null_without_a_device(driver):
    import orrery_b200 as ob

    ob.load_library()
    if ob.device_count() > 0:
        pytest.skip("a device is visible; the null case needs a machine without one")
    assert driver.try_create(False) == 0
    assert driver.try_create(True, "fp64") == 0


def test_device_integrator_refuses_a_host_field(driver, plummer):
    state, m = _state(plummer, 64)
    rc, _, _, _ = driver.run("reference-direct", state, m, 1e-3, 1, device_integrator=True)
    assert rc == -1
    assert "needs a B200DirectSolver or B200TreeSolver" in driver.last_error()


def test_driver_reference_runs_equal_the_reference_library(driver, reference, plummer):
    # The driver's own reference path against ref_shim's: same classes, same bits.
    state, m = _state(plummer, 256)
    rc, got, counts, name = driver.run("reference-direct", state, m, 1e-3, 5, method="yoshida4")
    assert rc == 0 and name == "direct"
    want = {k: state[k].copy() for k in state}
    exact = reference.direct(state["x"], state["y"], state["z"], m, 0.01)[0]
    want.update(ax=exact[:, 0].copy(), ay=exact[:, 1].copy(), az=exact[:, 2].copy())
    want = reference.integrate_direct(want, m, 0.01, 1e-3, 5, "yoshida4")
    assert all(np.array_equal(got[k], want[k]) for k in KEYS)
    assert counts == (16, 16 * 256 * 255, 0)


# ---------------------------------------------------------------- device

@pytest.mark.gpu
@pytest.mark.parametrize("method,steps", [("vv", 12), ("yoshida4", 6), ("rk4", 5)])
@pytest.mark.parametrize("device_integrator", [False, True])
def test_fp64_direct_runs_are_bit_identical(b200, driver, plummer, method, steps,
                                            device_integrator):
    state, m = _state(plummer, 1000)
    rc, want, want_counts, _ = driver.run("reference-direct", state, m, 1e-3, steps,
                                          method=method)
    assert rc == 0, driver.last_error()
    rc, got, counts, name = driver.run("b200-direct", state, m, 1e-3, steps, method=method,
                                       precision="fp64", device_integrator=device_integrator)
    assert rc == 0, driver.last_error()
    assert name == "b200-direct"
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k
    assert counts == want_counts


@pytest.mark.gpu
@pytest.mark.parametrize("method,steps", [("vv", 6), ("yoshida4", 3)])
@pytest.mark.parametrize("device_integrator", [False, True])
@pytest.mark.parametrize("quadrupole", [False, True])
def test_fp64_tree_runs_are_bit_identical(b200, driver, plummer, method, steps,
                                          device_integrator, quadrupole):
    state, m = _state(plummer)
    kw = dict(method=method, opening_angle=0.5, leaf_capacity=16, quadrupole=quadrupole)
    rc, want, want_counts, _ = driver.run("reference-tree", state, m, 1e-3, steps, **kw)
    assert rc == 0, driver.last_error()
    rc, got, counts, name = driver.run("b200-tree", state, m, 1e-3, steps, precision="fp64",
                                       device_integrator=device_integrator, **kw)
    assert rc == 0, driver.last_error()
    assert name == "b200-tree"
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k
    assert counts == want_counts


@pytest.mark.gpu
@pytest.mark.parametrize("field,precision,worst,rms", [
    ("direct", "fp32", 2e-4, 2e-5),   # the reference's FP32 CUDA bounds
    ("direct", "split", 2e-6, 2e-7),  # the precision form
    ("tree", "fp32", 1e-4, 1e-5),     # FP32 walk against the FP64 tree
])
def test_reduced_precision_fields_stay_within_their_bounds(b200, driver, plummer, field,
                                                           precision, worst, rms):
    state, m = _state(plummer)
    kw = dict(quadrupole=True) if field == "tree" else {}
    rc, want, _, _ = driver.run(f"reference-{field}", state, m, 1e-3, 0, **kw)
    assert rc == 0, driver.last_error()
    for device_integrator in (False, True):
        rc, got, counts, _ = driver.run(f"b200-{field}", state, m, 1e-3, 0, precision=precision,
                                        device_integrator=device_integrator, **kw)
        assert rc == 0, driver.last_error()
        a = np.stack([got[k] for k in ("ax", "ay", "az")], axis=1)
        a_ref = np.stack([want[k] for k in ("ax", "ay", "az")], axis=1)
        err = relative_errors(a, a_ref)
        assert err.max() < worst and np.sqrt(np.mean(err ** 2)) < rms, (err.max(), err.mean())
    # Ten Yoshida-4 steps through B200Integrator stay beside the reference's run.
    rc, want, _, _ = driver.run(f"reference-{field}", state, m, 1e-3, 10, method="yoshida4", **kw)
    rc2, got, counts, _ = driver.run(f"b200-{field}", state, m, 1e-3, 10, method="yoshida4",
                                     precision=precision, device_integrator=True, **kw)
    assert rc == 0 and rc2 == 0, driver.last_error()
    assert counts[0] == 1 + 10 * 3
    for k in ("x", "y", "z"):
        assert np.max(np.abs(got[k] - want[k])) < 1e-7 * np.max(np.abs(want[k]))
