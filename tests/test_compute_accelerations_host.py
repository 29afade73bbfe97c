"""The reference's call form of compute_accelerations on the CPU (no GPU).

``orrery.compute_accelerations(configuration, particles)``
(python/src/sim_bindings.cpp:383-410) reads only the configuration's solver
section, writes the particles' acceleration arrays in place and returns the
InteractionCount. Fake solvers stand in for the device, so what is checked
here is the mapping: which solver, which settings, which arrays.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

import orrery_b200 as ob


class Kind:
    """Stands in for the reference's SolverKind enum: str() gives the
    configuration file's spelling (src/sim/configuration.cpp:100-112)."""

    def __init__(self, text):
        self.text = text

    def __str__(self):
        return self.text


class FakeSolver:
    made = []

    def __init__(self, *args):
        self.args = args
        FakeSolver.made.append((type(self).__name__, args))

    def evaluate(self, positions, masses, accelerations=None):
        if accelerations is None:  # the array form: (N, 3) positions, a result
            return np.zeros_like(positions)
        x, y, z = positions
        for out, value in zip(accelerations, (x + masses, y * 2, -z)):
            out[...] = value

    def interaction_count(self):
        return ob.InteractionCount(1, 6, 0)


class FakeDirect(FakeSolver):
    pass


class FakeTree(FakeSolver):
    pass


@pytest.fixture
def fakes(monkeypatch):
    FakeSolver.made = []
    monkeypatch.setattr(ob, "B200DirectSolver", FakeDirect)
    monkeypatch.setattr(ob, "B200TreeSolver", FakeTree)
    return FakeSolver.made


def particles(n=3):
    rng = np.random.default_rng(2)
    p = SimpleNamespace(**{k: rng.standard_normal(n) for k in
                           ("position_x", "position_y", "position_z", "velocity_x",
                            "velocity_y", "velocity_z")})
    p.mass = np.full(n, 0.5)
    for k in ("acceleration_x", "acceleration_y", "acceleration_z"):
        setattr(p, k, np.zeros(n))
    return p


def configuration(kind, **solver):
    settings = dict(softening=0.02, opening_angle=0.7, leaf_capacity=16, quadrupole=True,
                    executor="work-stealing", threads=0)
    settings.update(solver)
    return SimpleNamespace(solver=SimpleNamespace(kind=Kind(kind), **settings))


@pytest.mark.parametrize("kind,made", [("direct", ("FakeDirect", (0.02, "fp64"))),
                                       ("sycl-direct", ("FakeDirect", (0.02, "fp64"))),
                                       ("barnes-hut", ("FakeTree", (0.02, 0.7, 16, True, "fp64"))),
                                       ("sycl-tree", ("FakeTree", (0.02, 0.7, 16, True, "fp64")))])
def test_the_solver_section_chooses_the_solver(fakes, kind, made):
    p = particles()
    count = ob.compute_accelerations(configuration(kind), p)
    assert fakes == [made]
    assert count == ob.InteractionCount(1, 6, 0)
    # Written in place, into the particles' own arrays.
    assert np.array_equal(p.acceleration_x, p.position_x + p.mass)
    assert np.array_equal(p.acceleration_y, p.position_y * 2)
    assert np.array_equal(p.acceleration_z, -p.position_z)


def test_precision_can_be_chosen(fakes):
    ob.compute_accelerations(configuration("direct"), particles(), precision="split")
    assert fakes == [("FakeDirect", (0.02, "split"))]


def test_an_unknown_kind_is_an_invalid_argument(fakes):
    with pytest.raises(ob.OrreryError) as e:
        ob.compute_accelerations(configuration("fmm"), particles())
    assert e.value.code == ob.ERROR_INVALID_ARGUMENT and fakes == []


def test_the_array_form_is_unchanged(fakes):
    p = particles()
    ob.compute_accelerations(np.stack([p.position_x, p.position_y, p.position_z], 1), p.mass,
                             softening=0.1, solver="tree")
    assert fakes == [("FakeTree", (0.1, 0.5, 32, False, "fp32"))]
