"""Checkpoints and trajectories of device-resident systems.

A system's checkpoint is byte-identical to the host writer's file of its
state (itself byte-identical to the reference's, tests/test_output_host.py);
a run resumed from a checkpoint continues bit for bit as the run that never
stopped (the reference's resume contract, tests/sim/simulation_test.cpp); and
trajectory frames snapshotted on the device while the system keeps stepping
hold exactly the states at those steps.
"""
from __future__ import annotations

import numpy as np
import pytest

from orrery_b200 import initial_conditions as ic

pytestmark = pytest.mark.gpu

ARRAYS = ("m", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def read_bytes(path):
    with open(path, "rb") as f:
        return f.read()


def make_system(b200, kind, n, seed=21):
    d = ic.plummer_sphere(n, seed=seed)
    if kind == "tree":
        s = b200.DeviceSystem(n, 0.02, b200.SOLVER_TREE, "fp32", 0.5, 32, True)
    else:
        s = b200.DeviceSystem(n, 0.01, b200.SOLVER_DIRECT, kind)
    s.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    return s, d


def full_state(system, masses):
    st = system.state()
    st["m"] = np.asarray(masses, dtype=np.float64)
    return st


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


def test_system_checkpoint_is_the_host_checkpoint_of_its_state(b200, tmp_path):
    s, d = make_system(b200, "fp64", 300)
    s.step(1e-3, 5, "vv")
    s.write_checkpoint(tmp_path / "dev.ck", 5, "[run]\ntimestep = 0.001\n")
    b200.write_checkpoint(tmp_path / "host.ck", 5, full_state(s, d["m"]),
                          "[run]\ntimestep = 0.001\n")
    assert read_bytes(tmp_path / "dev.ck") == read_bytes(tmp_path / "host.ck")
    back = b200.read_checkpoint(tmp_path / "dev.ck")
    st = full_state(s, d["m"])
    assert back["step"] == 5 and all(same_bits(back[k], st[k]) for k in ARRAYS)


@pytest.mark.parametrize("kind,integrator,n", [("fp64", "vv", 400), ("fp32", "yoshida4", 1000),
                                                ("split", "yoshida4", 700), ("tree", "vv", 5000),
                                                ("fp64", "rk4", 300), ("tree", "rk4", 3000)])
def test_resumed_run_continues_bit_for_bit(b200, tmp_path, kind, integrator, n):
    a, d = make_system(b200, kind, n)
    a.step(1e-3, 6, integrator)
    a.write_checkpoint(tmp_path / "run.ck", 6, "text")
    a.step(1e-3, 5, integrator)
    straight = a.state()

    b, _ = make_system(b200, kind, n, seed=99)  # different state, overwritten by the restore
    step, text = b.read_checkpoint(tmp_path / "run.ck")
    assert step == 6 and text == "text"
    b.step(1e-3, 5, integrator)
    resumed = b.state()
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        assert same_bits(straight[k], resumed[k]), k


def test_checkpoint_of_another_size_is_refused(b200, tmp_path):
    a, d = make_system(b200, "fp32", 100)
    a.write_checkpoint(tmp_path / "a.ck", 0)
    b, _ = make_system(b200, "fp32", 101)
    with pytest.raises(b200.OrreryError) as err:
        b.read_checkpoint(tmp_path / "a.ck")
    assert err.value.code == b200.ERROR_INVALID_ARGUMENT


@pytest.mark.parametrize("with_velocities", [False, True])
def test_device_trajectory_frames_are_the_states_at_their_steps(b200, tmp_path, with_velocities):
    n, dt = 2048, 1e-3
    s, d = make_system(b200, "fp32", n)
    twin, _ = make_system(b200, "fp32", n)
    path = tmp_path / "dev.tj"
    expected = []
    t = b200.Trajectory(path, dt, system=s, with_velocities=with_velocities)
    t.write_frame(0, 0.0)
    expected.append((0, 0.0, twin.state()))
    for k in range(1, 6):
        s.step_async(dt, 3, "vv")      # frames are taken between enqueued steps
        t.write_frame(3 * k, 3 * k * dt)
        twin.step(dt, 3, "vv")
        expected.append((3 * k, 3 * k * dt, twin.state()))
    s.step_async(dt, 2, "vv")          # steps after the last frame do not reach it
    t.close()
    s.synchronize()

    host = tmp_path / "host.tj"
    with b200.Trajectory(host, dt, masses=d["m"], with_velocities=with_velocities) as h:
        for step, time, st in expected:
            h.write_frame(step, time, st)
    assert read_bytes(path) == read_bytes(host)


def test_device_and_host_frames_share_one_ordered_file(b200, tmp_path):
    n, dt = 600, 1e-3
    s, d = make_system(b200, "fp64", n)
    path = tmp_path / "mixed.tj"
    t = b200.Trajectory(path, dt, system=s)
    first = s.state()
    t.write_frame(0, 0.0)
    s.step(dt, 2, "vv")
    second = s.state()
    t.write_frame(2, 2 * dt, second)   # host arrays through the same queue
    s.step(dt, 2, "vv")
    third = s.state()
    t.write_frame(4, 4 * dt)
    t.flush()
    assert t.frames == 3
    t.close()
    host = tmp_path / "host.tj"
    with b200.Trajectory(host, dt, masses=d["m"]) as h:
        for step, st in ((0, first), (2, second), (4, third)):
            h.write_frame(step, step * dt, st)
    assert read_bytes(path) == read_bytes(host)
