"""The synthetic-input samplers hold the reference's statistical checks.

initial_conditions.plummer_sphere restates the reference's Plummer sampler
(src/initial_conditions/plummer.cpp:43-128) with NumPy's generator in place of
mt19937_64, so a seed gives the same distribution rather than the same bits.
The claim is tested the way the reference tests its own sampler
(tests/initial_conditions/plummer_test.cpp:80-198): 4096 particles in the
standard model (M = 1, a = 3 pi / 16, so W = -1/2 and T = 1/4) are in virial
equilibrium within 0.10, have the model's energies within 8 %, are centred and
at rest to 64 machine epsilons, have the model's median radius 1.3048 a within
8 % and no particle beyond 40 a. The energies are measured by the reference's
own core::measure_diagnostics. Runs on the CPU.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from orrery_b200 import initial_conditions as ic

STANDARD_RADIUS = 3 * math.pi / 16
EPS = float(np.finfo(np.float64).eps)


@pytest.mark.parametrize("seed", [20260810, 1, 2, 3])
def test_a_sampled_plummer_sphere_is_the_models(reference, seed):
    a = STANDARD_RADIUS
    d = ic.plummer_sphere(4096, 1.0, a, seed=seed)
    g = reference.diagnostics(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"], 0.0)
    kinetic, potential = g["kinetic_energy"], g["potential_energy"]

    assert abs(2 * kinetic / abs(potential) - 1) <= 0.10             # virial equilibrium
    assert abs(potential - (-0.5)) <= 0.08 * 0.5                      # the model's energies
    assert abs(kinetic - 0.25) <= 0.08 * 0.25

    mass = math.fsum(d["m"])
    assert abs(mass - 1.0) <= 64 * EPS
    centre = math.hypot(*(math.fsum(d["m"] * d[k]) / mass for k in ("x", "y", "z")))
    assert centre <= 64 * EPS * a                                      # centred
    speed = math.sqrt(2 * kinetic / mass)
    assert np.linalg.norm(g["linear_momentum"]) <= 64 * EPS * mass * speed  # at rest

    radii = np.sort(np.sqrt(d["x"] ** 2 + d["y"] ** 2 + d["z"] ** 2))
    assert abs(radii[len(radii) // 2] - 1.3048 * a) <= 0.08 * 1.3048 * a
    assert radii[-1] <= 40 * a


def test_the_same_seed_samples_the_same_sphere():
    one, two = ic.plummer_sphere(500, seed=7), ic.plummer_sphere(500, seed=7)
    assert all(np.array_equal(one[k], two[k]) for k in one)
    other = ic.plummer_sphere(500, seed=8)
    assert not np.array_equal(one["x"], other["x"])


def test_a_plummer_sphere_shares_its_mass_equally_and_an_empty_one_is_empty():
    d = ic.plummer_sphere(1000, total_mass=3.0, seed=4)
    assert np.all(d["m"] == 3.0 / 1000)
    empty = ic.plummer_sphere(0)
    assert all(len(v) == 0 for v in empty.values())
