"""The device-resident Simulation against the reference's Simulation contract.

Restates the checks of the reference's Python suite
(python/tests/test_simulation.py): the clock is the step counter times the
timestep, a circular orbit closes after one period, a resumed run equals the
uninterrupted one in every bit. Adds the parts this backend provides: the
diagnostics equal core::measure_diagnostics bit for bit, run output at the
reference's record points (start, every stride, last step), and zero-copy
device views of the state.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from orrery_b200 import initial_conditions as ic

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def plummer(n, seed=3):
    return ic.plummer_sphere(n, seed=seed)


def circular_binary():
    # Equal masses 1 at separation 1, G = 1: relative speed sqrt(2), period
    # 2 pi / sqrt(2), each body at half the relative speed about the centre.
    v = math.sqrt(2.0) / 2.0
    return {"x": np.array([-0.5, 0.5]), "y": np.zeros(2), "z": np.zeros(2),
            "vx": np.zeros(2), "vy": np.array([-v, v]), "vz": np.zeros(2),
            "m": np.ones(2)}, 2.0 * math.pi / math.sqrt(2.0)


def test_the_clock_is_the_step_counter_times_the_timestep(b200):
    sim = b200.Simulation(plummer(256), timestep=1e-3, softening=0.01)
    assert sim.step_index == 0 and sim.time == 0.0
    sim.run(100)
    assert sim.step_index == 100
    assert sim.time == 100 * sim.timestep
    sim.step()
    assert sim.step_index == 101 and sim.time == 101 * 1e-3


@pytest.mark.parametrize("integrator", ["yoshida4", "rk4"])
def test_a_circular_orbit_returns_to_where_it_started(b200, integrator):
    state, period = circular_binary()
    sim = b200.Simulation(state, timestep=period / 512, integrator=integrator,
                          precision="fp64", softening=0.0)
    start = sim.particles
    sim.run(512)
    end = sim.particles
    for k in ("x", "y", "vx", "vy"):
        assert np.max(np.abs(end[k] - start[k])) < 1e-6, k


def test_measure_equals_the_reference_diagnostics(b200, reference):
    d = plummer(700, seed=8)
    sim = b200.Simulation(d, timestep=1e-3, softening=0.02, precision="fp64",
                          integrator="yoshida4")
    sim.run(5)
    st = sim.particles
    got = sim.measure()
    ref = reference.diagnostics(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"],
                                st["m"], 0.02)
    assert got["kinetic_energy"] == ref["kinetic_energy"]
    assert got["potential_energy"] == ref["potential_energy"]
    assert np.array_equal(got["linear_momentum"], ref["linear_momentum"])
    assert np.array_equal(got["angular_momentum"], ref["angular_momentum"])
    assert got["total_energy"] == got["kinetic_energy"] + got["potential_energy"]


def test_run_output_records_where_the_reference_does(b200, reference, tmp_path):
    # Frames at the first record, each multiple of the stride and the last
    # step (src/sim/run_output.cpp: due()); a checkpoint every 8 steps and at
    # the end.
    out = b200.FileOutput(trajectory_path=tmp_path / "run.tj", trajectory_stride=5,
                          trajectory_velocities=True, checkpoint_path=tmp_path / "run.ck",
                          checkpoint_stride=8, configuration="[run]\ntimestep = 0.001\n",
                          diagnostics_path=tmp_path / "run.csv", diagnostics_stride=5)
    sim = b200.Simulation(plummer(500), timestep=1e-3, softening=0.01, output=out)
    sim.run(23)
    out.close()
    got = reference.read_trajectory(tmp_path / "run.tj", max_frames=8, max_n=500)
    assert [f[0] for f in got["frames"]] == [0, 5, 10, 15, 20, 23]
    assert [f[1] for f in got["frames"]] == [s * 1e-3 for s in (0, 5, 10, 15, 20, 23)]
    final = sim.particles
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(got["frames"][-1][2][k], final[k])
    assert out.checkpoints == 4  # steps 0, 8, 16, 23
    ck = reference.read_checkpoint(tmp_path / "run.ck")
    assert ck["step"] == 23
    # The diagnostics rows fall on the frames' steps: the reference's
    # DiagnosticsLog over core::measure_diagnostics of each frame writes the
    # same file, byte for byte.
    rows = [(step, time, reference.diagnostics(st["x"], st["y"], st["z"], st["vx"], st["vy"],
                                               st["vz"], got["masses"], 0.01))
            for step, time, st in got["frames"]]
    reference.write_diagnostics_log(tmp_path / "ref.csv", rows)
    assert (tmp_path / "run.csv").read_bytes() == (tmp_path / "ref.csv").read_bytes()


@pytest.mark.parametrize("kind", ["direct", "barnes-hut"])
def test_compute_accelerations_in_the_reference_call_form(b200, reference, kind):
    # compute_accelerations(configuration, particles) writes the particles'
    # acceleration arrays in place and returns the count
    # (python/src/sim_bindings.cpp:383-410); at its default FP64 precision the
    # forces are the reference solvers' (scalar kernels) bit for bit.
    from types import SimpleNamespace

    d = plummer(900, seed=4)
    p = SimpleNamespace(position_x=d["x"].copy(), position_y=d["y"].copy(),
                        position_z=d["z"].copy(), mass=d["m"].copy(),
                        acceleration_x=np.zeros(900), acceleration_y=np.zeros(900),
                        acceleration_z=np.zeros(900))
    cfg = SimpleNamespace(solver=SimpleNamespace(kind=kind, softening=0.02, opening_angle=0.5,
                                                 leaf_capacity=32, quadrupole=True))
    count = b200.compute_accelerations(cfg, p)
    got = np.stack([p.acceleration_x, p.acceleration_y, p.acceleration_z], axis=1)
    if kind == "direct":
        want, pairs = reference.direct(d["x"], d["y"], d["z"], d["m"], 0.02)
        assert count.particle_particle == pairs
    else:
        want, counts, _ = reference.barnes_hut(d["x"], d["y"], d["z"], d["m"], 0.02, 0.5, 32,
                                               True, with_tree=False)
        assert (count.particle_particle, count.particle_cell) == (int(counts[1]),
                                                                  int(counts[2]))
    assert count.evaluations == 1
    assert np.array_equal(got, want)


def test_restore_takes_another_particle_count(b200, reference, tmp_path):
    # The reference's restore accepts any count (python/src/sim_bindings.cpp:
    # 293-309); its trajectory writer then skips frames of the wrong length
    # (src/sim/trajectory.cpp:73-79) while diagnostics rows go on.
    out = b200.FileOutput(trajectory_path=tmp_path / "t.tj", trajectory_stride=1,
                          diagnostics_path=tmp_path / "d.csv", diagnostics_stride=1)
    sim = b200.Simulation(plummer(300), timestep=1e-3, softening=0.01, precision="fp64",
                          output=out)
    sim.run(2)
    other = plummer(200, seed=9)
    sim.restore(other, step=2)
    assert sim.n == 200 and sim.step_index == 2
    sim.run(3)
    out.close()
    fresh = b200.Simulation(other, timestep=1e-3, softening=0.01, precision="fp64")
    fresh.run(3)
    got, want = sim.particles, fresh.particles
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k
    tj = reference.read_trajectory(tmp_path / "t.tj", max_frames=8, max_n=300)
    assert tj["n"] == 300 and [f[0] for f in tj["frames"]] == [0, 1, 2]
    rows = (tmp_path / "d.csv").read_text().splitlines()[1:]
    assert [int(r.split(",")[0]) for r in rows] == [0, 1, 2, 2, 3, 4, 5]


@pytest.mark.parametrize("solver,precision,integrator", [("direct", "fp32", "vv"),
                                                         ("tree", "fp32", "rk4"),
                                                         ("tree", "fp64", "yoshida4")])
def test_a_resumed_run_is_identical_in_every_bit(b200, tmp_path, solver, precision, integrator):
    d = plummer(2000, seed=12)
    kw = dict(timestep=1e-3, softening=0.02, solver=solver, precision=precision,
              integrator=integrator, quadrupole=True)
    straight = b200.Simulation(d, **kw)
    straight.run(10)
    first = b200.Simulation(d, **kw)
    first.run(6)
    first.write_checkpoint(tmp_path / "half.ck", "text")
    second = b200.Simulation(plummer(2000, seed=99), **kw)
    assert second.resume(tmp_path / "half.ck") == "text"
    assert second.step_index == 6
    second.run(4)
    a, b = straight.particles, second.particles
    assert second.time == straight.time
    assert all(np.array_equal(a[k], b[k]) for k in KEYS)


def test_restore_with_current_accelerations_evaluates_nothing(b200):
    d = plummer(300, seed=5)
    sim = b200.Simulation(d, timestep=1e-3, softening=0.01, precision="fp64")
    sim.run(3)
    st = sim.particles
    other = b200.Simulation(plummer(300, seed=6), timestep=1e-3, softening=0.01,
                            precision="fp64")
    before = other.interaction_count.evaluations
    other.restore(st, step=3, accelerations_are_current=True)
    assert other.interaction_count.evaluations == before
    assert other.step_index == 3
    sim.run(2)
    other.run(2)
    a, b = sim.particles, other.particles
    assert all(np.array_equal(a[k], b[k]) for k in KEYS)


def test_device_views_share_the_state_without_a_copy(b200):
    import torch
    d = plummer(1000, seed=2)
    sim = b200.Simulation(d, timestep=1e-3, softening=0.01)
    sim.run(2)
    views = sim.device_particles()
    x = torch.as_tensor(views["x"], device="cuda")
    m = torch.as_tensor(views["m"], device="cuda")
    host = sim.particles
    assert np.array_equal(x.cpu().numpy(), host["x"])
    assert np.array_equal(m.cpu().numpy(), host["m"])
    # A write through the view is the system's state.
    vx = torch.as_tensor(views["vx"], device="cuda")
    vx.zero_()
    torch.cuda.synchronize()
    assert not sim.particles["vx"].any()
    assert x.data_ptr() == views["x"].__cuda_array_interface__["data"][0]
