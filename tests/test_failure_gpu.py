"""Failure detection on the device without a GPU fault.

The library's device-side waits are bounded: a wait that runs out sets a bit
in the kernel's status word, the kernel returns, and the host reports
OB_ERROR_TIMEOUT after synchronising. Here a onesweep radix-sort pass runs
with its first tile never taken, so the look-back words its successors wait
on are never published; with a poll limit of a thousand the waits run out,
the call returns OB_ERROR_TIMEOUT, and the same process then sorts and
evaluates forces normally (the context stays usable). Nothing here faults,
traps or hangs the device: every wait ends after poll_limit polls.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry(b200):
    lib = b200.load_library()
    fn = lib.ob_test_lookback_timeout
    fn.argtypes = [C.c_uint64, C.c_uint32, C.c_int]
    fn.restype = C.c_int
    return lib, fn


def test_an_unpublished_lookback_times_out_and_the_device_stays_usable(b200, restatement):
    lib, fn = _entry(b200)
    assert fn(100_000, 1024, 1) == b200.ERROR_TIMEOUT
    assert b"look-back" in lib.ob_last_error()
    # The same pass with every tile present completes and sorts.
    assert fn(100_000, 1 << 24, 0) == b200.OK, lib.ob_last_error()
    # And the full pipeline still runs on this context.
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(3000, seed=77)
    solver = b200.B200TreeSolver(0.01, 0.5, 32, True)
    a = solver.evaluate((d["x"], d["y"], d["z"]), d["m"])
    a_ref, counts = restatement.barnes_hut(d["x"], d["y"], d["z"], d["m"], 0.01, 0.5, 32, True)
    c = solver.interaction_count()
    assert (c.particle_particle, c.particle_cell) == (counts.particle_particle,
                                                      counts.particle_cell)
    err = np.linalg.norm(a - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
    assert err.max() < 1e-4


def test_the_test_entry_checks_its_arguments(b200):
    lib, fn = _entry(b200)
    assert fn(0, 10, 0) == b200.ERROR_INVALID_ARGUMENT
    assert fn((1 << 24) + 1, 10, 0) == b200.ERROR_INVALID_ARGUMENT


@pytest.mark.parametrize("cap", [2, 24, 64])
def test_a_full_traversal_stack_falls_back_to_the_union_walk(b200, restatement, cap):
    # A stack capped at a few entries fills in (almost) every warp, which then
    # discards its partial sums and walks its targets one by one: the
    # counters must still be the reference's and the forces within the
    # tree's bounds, whichever warps fell back.
    from orrery_b200 import initial_conditions as ic
    lib = b200.load_library()
    lib.ob_test_set_walk_stack_cap.argtypes = [C.c_void_p, C.c_uint32]
    lib.ob_test_set_walk_stack_cap.restype = C.c_int
    d = ic.galaxy_collision(20_000, softening=0.02, seed=31)
    x, y, z, m = d["x"], d["y"], d["z"], d["m"]
    a_ref, counts = restatement.barnes_hut(x, y, z, m, 0.02, 0.5, 32, True)
    solver = b200.B200TreeSolver(0.02, 0.5, 32, True)
    assert lib.ob_test_set_walk_stack_cap(solver._handle, cap) == b200.OK
    a = solver.evaluate((x, y, z), m)
    c = solver.interaction_count()
    assert (c.particle_particle, c.particle_cell) == (counts.particle_particle,
                                                      counts.particle_cell)
    err = np.linalg.norm(a - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
    assert err.max() < 1e-4 and np.sqrt(np.mean(err ** 2)) < 1e-5
    # Back to the full stack: the same counts.
    assert lib.ob_test_set_walk_stack_cap(solver._handle, 0) == b200.OK
    solver.reset_interaction_count()
    solver.evaluate((x, y, z), m)
    c2 = solver.interaction_count()
    assert (c2.particle_particle, c2.particle_cell) == (counts.particle_particle,
                                                        counts.particle_cell)


def test_the_stack_cap_is_refused_where_it_does_not_apply(b200):
    lib = b200.load_library()
    lib.ob_test_set_walk_stack_cap.argtypes = [C.c_void_p, C.c_uint32]
    direct = b200.B200DirectSolver(0.01)
    assert lib.ob_test_set_walk_stack_cap(direct._handle, 8) == b200.ERROR_UNSUPPORTED
    tree = b200.B200TreeSolver(0.01, 0.5, 32, True)
    assert lib.ob_test_set_walk_stack_cap(tree._handle, 257) == b200.ERROR_INVALID_ARGUMENT


def test_a_fused_launch_whose_ready_word_never_comes_times_out(b200):
    # The fused small-system launch waits for each CTA's ready word; with one
    # CTA silent and a poll limit of a thousand the waits run out, the step
    # reports OB_ERROR_TIMEOUT, and the next launch (ready words cleared)
    # steps exactly as a fresh system does.
    from orrery_b200 import initial_conditions as ic
    lib = b200.load_library()
    lib.ob_test_fused_timeout.argtypes = [C.c_void_p, C.c_uint32]
    lib.ob_test_fused_timeout.restype = C.c_int
    d = ic.plummer_sphere(2048, seed=12)
    keys = ("x", "y", "z", "vx", "vy", "vz", "m")

    def fresh():
        s = b200.DeviceSystem(2048, 0.01, precision="fp32")
        assert s.set_fused_steps(True)
        s.set_state(*(d[k] for k in keys))
        return s

    s = fresh()
    assert lib.ob_test_fused_timeout(s._handle, 1000) == b200.OK
    with pytest.raises(b200.OrreryError) as err:
        s.step(1e-3, 3, "vv")
    assert err.value.code == b200.ERROR_TIMEOUT
    s.set_state(*(d[k] for k in keys))
    s.step(1e-3, 5, "vv")
    reference = fresh()
    reference.step(1e-3, 5, "vv")
    a, b = s.state(), reference.state()
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        assert np.array_equal(a[k], b[k]), k


def test_the_fused_timeout_entry_checks_its_arguments(b200):
    lib = b200.load_library()
    lib.ob_test_fused_timeout.argtypes = [C.c_void_p, C.c_uint32]
    lib.ob_test_fused_timeout.restype = C.c_int
    big = b200.DeviceSystem(100_000, 0.01, precision="fp32")
    assert lib.ob_test_fused_timeout(big._handle, 10) == b200.ERROR_UNSUPPORTED
    small = b200.DeviceSystem(512, 0.01, precision="fp32")
    assert lib.ob_test_fused_timeout(small._handle, 0) == b200.ERROR_INVALID_ARGUMENT
