"""A run on the device: the counterpart of the reference's sim::Simulation and
its run output, over the C ABI.

``Simulation`` mirrors the reference's Python ``orrery.Simulation``
(python/src/sim_bindings.cpp:274-343, src/sim/simulation.cpp:16-70): it holds
the state, the solver, the integrator and the step counter; the simulated time
is ``step_index * timestep``, computed rather than accumulated; ``run`` records
through an attached output at the start, every stride and the last step, as
sim::FileOutput::record does (src/sim/run_output.cpp). The state stays in HBM:
``particles`` copies it to the host, ``device_particles`` gives zero-copy views
of it (``__cuda_array_interface__``, readable by torch, CuPy or Numba).
"""
from __future__ import annotations

import collections
import ctypes as C
import math

import numpy as np

from . import (DeviceSystem, OrreryError, Trajectory, SOLVER_DIRECT, SOLVER_TREE,
               ERROR_INVALID_ARGUMENT, INTEGRATOR_RK4, INTEGRATOR_VV, INTEGRATOR_YOSHIDA4,
               _INTEGRATORS, _PARTICLE_NAMES, _check, _count, _f64, _ptr, _state_of,
               load_library)

_STATE = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")

# Integrator::name of the reference's three integrators
# (include/orrery/integrators/{velocity_verlet,yoshida4,runge_kutta4}.hpp).
_INTEGRATOR_NAMES = {INTEGRATOR_VV: "velocity Verlet", INTEGRATOR_YOSHIDA4: "Yoshida 4",
                     INTEGRATOR_RK4: "RK4"}


class DeviceArrayView:
    """One FP64 state array of a DeviceSystem, exposed without a copy through
    ``__cuda_array_interface__`` (version 3). Valid while the system lives;
    reads and writes from another stream must be ordered against the
    system's steps by the caller (``DeviceSystem.synchronize``)."""

    def __init__(self, address: int, n: int, owner):
        self._owner = owner  # keeps the system alive
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8",
                                         "data": (address, False), "version": 3,
                                         "strides": None, "stream": None}

    def __len__(self):
        return self.__cuda_array_interface__["shape"][0]


def device_arrays(system: DeviceSystem) -> dict:
    """Zero-copy views of a system's ten state arrays, keyed x y z vx vy vz ax
    ay az m (ob_system_device_arrays)."""
    lib = load_library()
    ptrs = (C.c_void_p * 10)()
    _check(lib.ob_system_device_arrays(system._handle, ptrs))
    return {k: DeviceArrayView(ptrs[i] or 0, system.n, system) for i, k in enumerate(_STATE)}


_DIAGNOSTICS_HEADER = ("step,time,kinetic_energy,potential_energy,total_energy,"
                       "relative_energy_error,virial_ratio,momentum_x,momentum_y,momentum_z,"
                       "angular_momentum_x,angular_momentum_y,angular_momentum_z\n")


def _real(value: float) -> str:
    """A double as the reference's log writes it: an ostream in the classic
    locale at max_digits10 = 17 significant digits, i.e. C's "%.17g", whose
    NaN carries its sign ("-nan" for the x86 default NaN of 0/0)."""
    if value != value:
        return "-nan" if math.copysign(1.0, value) < 0 else "nan"
    return "%.17g" % value


def _virial_ratio(kinetic: float, potential: float) -> float:
    """2T/|U| with IEEE division (core/diagnostics.hpp:79-82): no potential
    energy gives an infinity, or a NaN when nothing moves either."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return float(np.float64(2 * kinetic) /
                     np.float64(-potential if potential < 0 else potential))


Vec3 = collections.namedtuple("Vec3", "x y z")
Vec3.__doc__ = """A momentum as the reference's Python Vec3 gives it: x, y, z by name,
a sequence of three (unpacking, tuple(), numpy.asarray())."""


class Diagnostics(dict):
    """core::Diagnostics as the reference's Python binding exposes it
    (python/src/core_bindings.cpp:139-158): kinetic_energy, potential_energy,
    linear_momentum and angular_momentum, and the derived total_energy and
    virial_ratio, read as attributes; the same values by key."""

    def __getattr__(self, name):
        try:
            return self[name]
        except KeyError:
            raise AttributeError(name) from None

    def __repr__(self):
        return ("Diagnostics(" + ", ".join(f"{k}={_real(self[k])}" for k in (
            "kinetic_energy", "potential_energy", "total_energy", "virial_ratio")) + ")")


class Particles(dict):
    """A host copy of a simulation's state: arrays by key (x y z vx vy vz ax
    ay az m), or by the names of the reference's ParticleData (position_x ...
    acceleration_z, mass, and size)."""

    def __getattr__(self, name):
        key = _PARTICLE_NAMES.get(name)
        if key is not None:
            return self[key]
        if name == "size":
            return len(self["m"])
        raise AttributeError(name)


class DiagnosticsLog:
    """sim::DiagnosticsLog (src/sim/diagnostics_log.cpp): a CSV of the
    conserved quantities, one row per measurement, every number at full
    precision. The first row fixes the energy the error column is relative to
    (core::relative_energy_error, src/core/diagnostics.cpp:85-89: the absolute
    difference when that energy is zero)."""

    def __init__(self, path):
        self._file = open(path, "w", encoding="ascii", newline="\n")
        self._file.write(_DIAGNOSTICS_HEADER)
        self.reference_energy = None

    def record(self, step: int, time: float, diagnostics: dict) -> None:
        kinetic = float(diagnostics["kinetic_energy"])
        potential = float(diagnostics["potential_energy"])
        energy = kinetic + potential
        if self.reference_energy is None:
            self.reference_energy = energy
        scale = abs(self.reference_energy)
        difference = energy - self.reference_energy
        error = difference / scale if scale > 0 else difference
        row = [kinetic, potential, energy, error, _virial_ratio(kinetic, potential),
               *(float(v) for v in diagnostics["linear_momentum"]),
               *(float(v) for v in diagnostics["angular_momentum"])]
        self._file.write(f"{int(step)},{_real(float(time))}," +
                         ",".join(_real(v) for v in row) + "\n")

    def flush(self) -> None:
        self._file.flush()

    def close(self) -> None:
        self._file.close()


class FileOutput:
    """sim::FileOutput (src/sim/run_output.cpp): a trajectory frame every
    ``trajectory_stride`` steps, a diagnostics row every ``diagnostics_stride``
    and a checkpoint every ``checkpoint_stride``, each also at the first record
    and the last step of a run (a stride of 0: only those). Frames are device
    snapshots written in the background. The trajectory and the diagnostics
    log are flushed with each checkpoint, after it is written, as the
    reference does."""

    def __init__(self, trajectory_path=None, trajectory_stride: int = 0,
                 trajectory_velocities: bool = False, checkpoint_path=None,
                 checkpoint_stride: int = 0, configuration: str = "",
                 diagnostics_path=None, diagnostics_stride: int = 0):
        self.trajectory_path = trajectory_path
        self.trajectory_stride = int(trajectory_stride)
        self.trajectory_velocities = bool(trajectory_velocities)
        self.checkpoint_path = checkpoint_path
        self.checkpoint_stride = int(checkpoint_stride)
        self.diagnostics_path = diagnostics_path
        self.diagnostics_stride = int(diagnostics_stride)
        self.configuration = configuration
        self._trajectory = None
        self._diagnostics = None
        self._first = True
        self.checkpoints = 0

    def _due(self, step, stride, is_final):
        return self._first or is_final or (stride != 0 and step % stride == 0)

    def next_due(self, step: int, last: int) -> int:
        """The first step after `step`, up to `last`, at which something is due."""
        due = last
        for stride, on in ((self.trajectory_stride, self.trajectory_path),
                           (self.diagnostics_stride, self.diagnostics_path),
                           (self.checkpoint_stride, self.checkpoint_path)):
            if on and stride > 0:
                due = min(due, (step // stride + 1) * stride)
        return due

    def record(self, simulation: "Simulation", is_final: bool) -> None:
        step = simulation.step_index
        if self.trajectory_path is not None:
            if self._trajectory is None:
                self._trajectory = Trajectory(self.trajectory_path, simulation.timestep,
                                              system=simulation.system,
                                              with_velocities=self.trajectory_velocities)
            if self._due(step, self.trajectory_stride, is_final):
                if self._trajectory._system is simulation.system:
                    self._trajectory.write_frame(step, simulation.time)
                elif simulation.n == self._trajectory.n:
                    # The system was replaced by a restore: a frame of its state
                    # from the host.
                    self._trajectory.write_frame(step, simulation.time, simulation.particles)
                # A state of another particle count is not written: the format
                # has no per-frame length (src/sim/trajectory.cpp:73-79).
        if self.diagnostics_path is not None:
            if self._diagnostics is None:
                self._diagnostics = DiagnosticsLog(self.diagnostics_path)
            if self._due(step, self.diagnostics_stride, is_final):
                self._diagnostics.record(step, simulation.time, simulation.measure())
        if self.checkpoint_path is not None and \
                self._due(step, self.checkpoint_stride, is_final):
            simulation.write_checkpoint(self.checkpoint_path, self.configuration)
            self.checkpoints += 1
            if self._trajectory is not None:
                self._trajectory.flush()
            if self._diagnostics is not None:
                self._diagnostics.flush()
        self._first = False

    @property
    def frames_written(self) -> int:
        return self._trajectory.frames if self._trajectory is not None else 0

    def close(self) -> None:
        if self._trajectory is not None:
            self._trajectory.close()
            self._trajectory = None
        if self._diagnostics is not None:
            self._diagnostics.close()
            self._diagnostics = None


class Simulation:
    """sim::Simulation with its state resident on the device.

    ``state`` holds x y z vx vy vz m (FP64 arrays of one length). Building it
    costs one force evaluation, which establishes the carried accelerations
    (the reference's constructor does the same, src/sim/simulation.cpp:23)."""

    def __init__(self, state: dict, timestep: float, integrator: str = "vv",
                 solver: str = "direct", precision: str = "fp32", softening: float = 0.0,
                 opening_angle: float = 0.5, leaf_capacity: int = 32,
                 quadrupole: bool = False, output: FileOutput = None):
        kind = SOLVER_TREE if solver in ("tree", "barnes-hut") else SOLVER_DIRECT
        if solver not in ("direct", "tree", "barnes-hut"):
            raise OrreryError(ERROR_INVALID_ARGUMENT, f"unknown solver {solver!r}")
        if integrator not in _INTEGRATORS:
            raise OrreryError(ERROR_INVALID_ARGUMENT, f"unknown integrator {integrator!r}")
        state = _state_of(state)
        arrs = {k: _f64(state[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        self.n = len(arrs["m"])
        self._solver = (softening, kind, precision, opening_angle, leaf_capacity, quadrupole)
        self.system = DeviceSystem(self.n, *self._solver)
        self.system.set_state(arrs["x"], arrs["y"], arrs["z"], arrs["vx"], arrs["vy"],
                              arrs["vz"], arrs["m"])
        self.timestep = float(timestep)
        self._integrator = integrator
        self.solver_name = "b200-tree" if kind == SOLVER_TREE else "b200-direct"
        self.output = output
        self._step = 0

    @property
    def integrator_name(self) -> str:
        """The integrator's name as the reference's integrators give it
        (Integrator::name: "velocity Verlet", "Yoshida 4", "RK4")."""
        return _INTEGRATOR_NAMES[_INTEGRATORS[self._integrator]]

    # -- the clock ----------------------------------------------------------

    @property
    def step_index(self) -> int:
        return self._step

    @property
    def time(self) -> float:
        """The simulated time, step_index * timestep (computed, not accumulated)."""
        return float(self._step) * self.timestep

    # -- stepping -----------------------------------------------------------

    def step(self) -> None:
        """Advance by one step. Records nothing."""
        self.system.step(self.timestep, 1, self._integrator)
        self._step += 1

    def run(self, steps: int) -> None:
        """Advance by `steps` steps, recording through the output (if any) at
        the start, wherever a stride falls and at the last step."""
        steps = _count(steps, "steps")
        out = self.output
        if out is None:
            self.system.step(self.timestep, steps, self._integrator)
            self._step += steps
            return
        out.record(self, steps == 0)
        end = self._step + steps
        while self._step < end:
            target = out.next_due(self._step, end)
            self.system.step_async(self.timestep, target - self._step, self._integrator)
            self._step = target
            out.record(self, self._step == end)
        self.system.synchronize()

    # -- state --------------------------------------------------------------

    @property
    def particles(self) -> "Particles":
        """A host copy of the state, read by key (x y z vx vy vz ax ay az m) or
        by the reference's names (position_x ... acceleration_z, mass)."""
        return Particles(self.system.snapshot())

    def device_particles(self) -> dict:
        """Zero-copy views of the device state (see DeviceArrayView)."""
        self.system.synchronize()
        return device_arrays(self.system)

    def restore(self, state: dict, step: int = 0, accelerations_are_current: bool = False):
        """Replace the state and the step counter. Re-establishes the carried
        accelerations with one evaluation unless they are given as current.
        The particle count may differ from the current one
        (python/src/sim_bindings.cpp:293-309): the state then moves to a new
        device system of that size, with the same solver settings."""
        keys = ("x", "y", "z", "vx", "vy", "vz", "m")
        state = _state_of(state)
        arrs = {k: _f64(state[k]) for k in keys}
        n = len(arrs["m"])
        if any(len(a) != n for a in arrs.values()):
            raise OrreryError(ERROR_INVALID_ARGUMENT, "the state arrays differ in length")
        if n != self.n:
            self.system = DeviceSystem(n, *self._solver)
            self.n = n
        if accelerations_are_current:
            acc = {k: _f64(state[k]) for k in ("ax", "ay", "az")}
            lib = load_library()
            _check(lib.ob_system_restore(self.system._handle, _ptr(arrs["m"]),
                                         *(_ptr(arrs[k]) for k in keys[:6]),
                                         *(_ptr(acc[k]) for k in ("ax", "ay", "az"))))
        else:
            self.system.set_state(*(arrs[k] for k in keys))
        self._step = _count(step, "step")

    def measure(self) -> "Diagnostics":
        """core::measure_diagnostics of the current state: kinetic, potential
        and total energy, linear and angular momentum, virial ratio."""
        d = self.system.diagnostics()
        kinetic, potential = float(d["kinetic_energy"]), float(d["potential_energy"])
        return Diagnostics(kinetic_energy=kinetic, potential_energy=potential,
                           linear_momentum=Vec3(*(float(v) for v in d["linear_momentum"])),
                           angular_momentum=Vec3(*(float(v) for v in d["angular_momentum"])),
                           total_energy=kinetic + potential,
                           virial_ratio=_virial_ratio(kinetic, potential))

    @property
    def interaction_count(self):
        return self.system.interaction_count()

    # -- checkpoints --------------------------------------------------------

    def write_checkpoint(self, path, configuration: str = "") -> None:
        self.system.write_checkpoint(path, self._step, configuration)

    def resume(self, path) -> str:
        """Restore from an ORRERYCK checkpoint of this size (state, carried
        accelerations and step); returns its configuration text."""
        step, text = self.system.read_checkpoint(path)
        self._step = step
        return text

    def __repr__(self):
        return f"<Simulation of {self.n} particles at step {self._step}>"
