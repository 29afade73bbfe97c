"""The run loop's record points on the CPU (no GPU): sim::FileOutput::record
(src/sim/run_output.cpp) records at the first call, wherever a stride falls
and at the last step of a run; Simulation.run steps the device from one such
point to the next. A stub system stands in for the device."""
from __future__ import annotations

import orrery_b200 as ob
from orrery_b200.simulation import FileOutput, Simulation


class StubSystem:
    def __init__(self):
        self.enqueued = []

    def step_async(self, dt, steps, integrator):
        self.enqueued.append(steps)

    def step(self, dt, steps, integrator):
        self.enqueued.append(steps)

    def synchronize(self):
        pass

    def write_checkpoint(self, path, step, configuration=""):
        self.last_checkpoint = (path, step, configuration)

    def set_state(self, *arrays):
        self.state = arrays

    def snapshot(self):
        keys = ("m", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
        return {k: [float(i)] * 2 for i, k in enumerate(keys)}

    def diagnostics(self):
        return {"kinetic_energy": 0.25, "potential_energy": -0.5,
                "linear_momentum": [0.0, 0.0, 0.0], "angular_momentum": [0.0, 0.0, 1.0]}


def stub_simulation(output):
    sim = Simulation.__new__(Simulation)  # no device: only the loop is exercised
    sim.system = StubSystem()
    sim.timestep = 1e-3
    sim._integrator = "vv"
    sim.output = output
    sim._step = 0
    sim.n = 0
    return sim


class Recorder(FileOutput):
    def __init__(self, **kw):
        super().__init__(**kw)
        self.points = []

    def record(self, simulation, is_final):
        self.points.append((simulation.step_index, is_final))
        super().record(simulation, is_final)


def test_checkpoints_fall_at_start_strides_and_end():
    out = Recorder(checkpoint_path="run.ck", checkpoint_stride=8, configuration="text")
    sim = stub_simulation(out)
    sim.run(23)
    assert [p for p, _ in out.points] == [0, 8, 16, 23]
    assert out.points[-1] == (23, True)
    assert out.checkpoints == 4
    assert sim.system.last_checkpoint == ("run.ck", 23, "text")
    assert sum(sim.system.enqueued) == 23 and sim.step_index == 23
    assert sim.time == 23 * 1e-3


def test_a_second_run_continues_the_strides():
    out = Recorder(checkpoint_path="run.ck", checkpoint_stride=10)
    sim = stub_simulation(out)
    sim.run(12)
    sim.run(15)
    # The first call records step 0; the second run starts at 12 and records
    # 20, then its last step 27 (src/sim/simulation.cpp:52-64).
    assert [p for p, _ in out.points] == [0, 10, 12, 12, 20, 27]
    assert sim.step_index == 27


def test_diagnostics_rows_fall_at_start_strides_and_end(tmp_path):
    path = tmp_path / "run.csv"
    out = Recorder(diagnostics_path=path, diagnostics_stride=4)
    sim = stub_simulation(out)
    sim.run(10)
    out.close()
    lines = path.read_text().splitlines()
    assert lines[0].startswith("step,time,kinetic_energy,")
    assert [int(r.split(",")[0]) for r in lines[1:]] == [0, 4, 8, 10]
    assert [float(r.split(",")[1]) for r in lines[1:]] == [0.0, 4e-3, 8e-3, 10 * 1e-3]
    # The device was stepped only to the record points.
    assert sim.system.enqueued == [4, 4, 2]


def test_next_due_takes_the_nearest_stride():
    out = FileOutput(trajectory_path="t", trajectory_stride=5, checkpoint_path="c",
                     checkpoint_stride=8)
    assert out.next_due(0, 100) == 5
    assert out.next_due(5, 100) == 8
    assert out.next_due(8, 100) == 10
    assert out.next_due(39, 40) == 40
    assert FileOutput().next_due(3, 50) == 50
    assert FileOutput(diagnostics_path="d", diagnostics_stride=3).next_due(3, 50) == 6


def test_a_negative_run_is_refused_before_anything_is_enqueued():
    import pytest

    sim = stub_simulation(Recorder(checkpoint_path="c", checkpoint_stride=2))
    with pytest.raises(ob.OrreryError, match="must be in"):
        sim.run(-3)
    assert sim.system.enqueued == [] and sim.output.points == [] and sim.step_index == 0


def test_a_run_without_output_is_one_enqueue():
    sim = stub_simulation(None)
    sim.run(17)
    assert sim.system.enqueued == [17] and sim.step_index == 17


def test_virial_ratio_follows_the_reference_division():
    # 2T/|U| (core/diagnostics.hpp:79-82): a bound state gives a number, no
    # potential energy an infinity, and nothing at all a NaN.
    import math

    sim = stub_simulation(None)
    for kinetic, potential, expected in ((0.25, -0.5, 1.0), (0.5, 0.0, math.inf),
                                         (0.0, 0.0, math.nan), (0.125, 0.5, 0.5)):
        sim.system.diagnostics = lambda k=kinetic, p=potential: {
            "kinetic_energy": k, "potential_energy": p, "linear_momentum": [0.0] * 3,
            "angular_momentum": [0.0] * 3}
        d = sim.measure()
        assert d["total_energy"] == kinetic + potential
        if math.isnan(expected):
            assert math.isnan(d["virial_ratio"])
        else:
            assert d["virial_ratio"] == expected


def test_measure_reads_as_the_references_diagnostics():
    # core::Diagnostics through the reference's binding
    # (python/src/core_bindings.cpp:139-158): attributes, derived properties,
    # momenta as (x, y, z) vectors; the same values by key.
    import numpy as np

    d = stub_simulation(None).measure()
    assert isinstance(d, ob.Diagnostics)
    assert (d.kinetic_energy, d.potential_energy) == (0.25, -0.5)
    assert d.total_energy == -0.25 and d.virial_ratio == 1.0
    x, y, z = d.angular_momentum
    assert (x, y, z) == (0.0, 0.0, 1.0) and d.angular_momentum.z == 1.0
    assert np.array_equal(np.asarray(d.linear_momentum), np.zeros(3))
    assert d["total_energy"] == d.total_energy
    assert repr(d) == ("Diagnostics(kinetic_energy=0.25, potential_energy=-0.5, "
                       "total_energy=-0.25, virial_ratio=1)")
    import pytest
    with pytest.raises(AttributeError):
        d.energy


def test_particles_read_by_the_references_names():
    p = stub_simulation(None).particles
    assert isinstance(p, ob.Particles)
    assert p.mass == p["m"] == [0.0, 0.0] and p.position_y == p["y"] == [2.0, 2.0]
    assert p.acceleration_z == p["az"] and p.velocity_x == p["vx"] and p.size == 2


def test_restore_takes_the_references_particle_data():
    # ParticleData (python/src/core_bindings.cpp:241-300) as the reference's
    # restore takes it; a dict keyed x ... m as before.
    from types import SimpleNamespace

    import numpy as np

    sim = stub_simulation(None)
    sim.n = 2
    names = ("position_x", "position_y", "position_z", "velocity_x", "velocity_y",
             "velocity_z", "mass")
    data = SimpleNamespace(**{k: np.full(2, float(i)) for i, k in enumerate(names)})
    sim.restore(data, step=5)
    assert [a[0] for a in sim.system.state] == [0.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0]
    assert sim.step_index == 5
    import pytest
    with pytest.raises(ob.OrreryError):
        sim.restore(SimpleNamespace(position_x=[1.0]))


def test_integrator_names_are_the_reference_integrators_names():
    # Integrator::name (include/orrery/integrators/*.hpp), whichever of the
    # configuration's spellings chose it.
    sim = stub_simulation(None)
    for key, name in (("vv", "velocity Verlet"), ("velocity-verlet", "velocity Verlet"),
                      ("yoshida4", "Yoshida 4"), ("rk4", "RK4"), ("runge-kutta4", "RK4")):
        sim._integrator = key
        assert sim.integrator_name == name


def test_an_unknown_integrator_is_refused_before_the_device_is_touched():
    import pytest

    with pytest.raises(ob.OrreryError):
        Simulation({"m": [1.0]}, timestep=1e-3, integrator="euler")


def test_the_package_exports_the_run_surface():
    assert ob.Simulation is Simulation and ob.FileOutput is FileOutput
