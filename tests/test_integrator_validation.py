"""The reference's integrator validation, restated, with its published figures.

The reference validates its integrators on Kepler orbits
(tests/integrators/convergence_test.cpp, energy_behaviour_test.cpp) and
publishes what they measure (docs/validation.md:114-143):

* convergence order on a circular orbit closed after one period: velocity
  Verlet 1.9998, Yoshida-4 4.0006, RK4 4.1670;
* the energy envelope of an eccentric orbit (e = 0.5, 200 steps an orbit, 400
  orbits, sampled every 10 steps): velocity Verlet 2.6894e-3 in the first and
  the last twentieth, Yoshida-4 2.0170e-5 in both, RK4 1.92e-5 growing to
  3.72e-4.

Here the C restatement (the oracle) reproduces those figures to the digits
printed, on orbits from this package's Kepler generator, which is the
reference's bit for bit; tests/test_system_gpu.py makes the same runs on the
device. Runs on the CPU.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from orrery_b200 import initial_conditions as ic

STEPS_PER_ORBIT = 200
ORBITS = 400
SAMPLE_EVERY = 10

# docs/validation.md:116-118 and 141-143.
PUBLISHED_ORDERS = {"vv": "1.9998", "yoshida4": "4.0006", "rk4": "4.1670"}
PUBLISHED_ENVELOPES = {"vv": ("2.6894e-03", "2.6894e-03", 5),
                       "yoshida4": ("2.0170e-05", "2.0170e-05", 5),
                       "rk4": ("1.92e-05", "3.72e-04", 3)}


def envelope(step_chunk, energy, total=ORBITS * STEPS_PER_ORBIT):
    """energy_behaviour_test.cpp:integrate: the largest relative energy error
    over the first and the last twentieth of the run, and over all of it."""
    e0 = energy()
    window = total // 20
    early = late = extreme = 0.0
    done = 0
    while done < total:
        step_chunk(SAMPLE_EVERY)
        done += SAMPLE_EVERY
        error = abs((energy() - e0) / e0)
        extreme = max(extreme, error)
        if done - 1 < window:
            early = max(early, error)
        if done - 1 >= total - window:
            late = max(late, error)
    return early, late, extreme


def check_envelope(integrator, early, late, extreme):
    want_early, want_late, digits = PUBLISHED_ENVELOPES[integrator]
    fmt = f"{{:.{digits - 1}e}}"
    assert (fmt.format(early), fmt.format(late)) == (want_early, want_late)
    if integrator == "rk4":
        assert late >= 10 * early  # energy_behaviour_test.cpp: RK4 loses energy without bound
    else:
        assert extreme <= 0.005 and late <= 2 * early  # the symplectic envelope


def closure_order(closure, coarse):
    """convergence_test.cpp: log2 of the closure errors after one period at
    `coarse` and 2 `coarse` steps."""
    c, f = closure(coarse), closure(2 * coarse)
    assert 0 < f < c
    return math.log2(c / f)


COARSE = {"vv": 256, "yoshida4": 128, "rk4": 128}


class OracleOrbit:
    def __init__(self, restatement, orbit, timestep, integrator):
        self.r, self.dt, self.integrator = restatement, timestep, integrator
        self.m = orbit["m"]
        s = {k: orbit[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz")}
        a, _ = restatement.direct(s["x"], s["y"], s["z"], self.m, 0.0)
        s.update(ax=a[:, 0].copy(), ay=a[:, 1].copy(), az=a[:, 2].copy())
        self.s = s

    def step(self, steps):
        self.s, _ = self.r.integrate_direct(self.s, self.m, 0.0, self.dt, steps, self.integrator)

    def energy(self):
        s = self.s
        return (self.r.kinetic_energy(s["vx"], s["vy"], s["vz"], self.m) +
                self.r.potential_energy(s["x"], s["y"], s["z"], self.m, 0.0))


@pytest.mark.parametrize("params", [(1.0, 1.0, 1.0, 0.0), (1.0, 1.0, 1.0, 0.5),
                                    (2.0, 1.0, 1.5, 0.5), (1.0, 1e-3, 5.2, 0.0489),
                                    (0.3, 0.7, 0.01, 0.999)])
def test_kepler_orbit_is_the_references(reference, params):
    want, period = reference.kepler_orbit(*params)
    got = ic.kepler_orbit(*params)
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        assert np.array_equal(got[k], want[k]), k
    assert ic.kepler_period(*params) == period


@pytest.mark.parametrize("params", [(0.0, 1.0, 1.0, 0.0), (1.0, -1.0, 1.0, 0.0),
                                    (1.0, 1.0, 0.0, 0.0), (1.0, 1.0, 1.0, 1.0),
                                    (1.0, 1.0, 1.0, -0.1), (math.nan, 1.0, 1.0, 0.0),
                                    (1.0, 1.0, 1.0, math.nan)])
def test_unbound_or_invalid_orbits_are_refused_as_the_reference_refuses(reference, params):
    assert reference.kepler_orbit(*params) is None
    with pytest.raises(ValueError):
        ic.kepler_orbit(*params)
    with pytest.raises(ValueError):
        ic.kepler_period(*params)


@pytest.mark.parametrize("integrator", ["vv", "yoshida4", "rk4"])
def test_the_oracle_converges_at_the_published_orders(restatement, integrator):
    def closure(steps):
        start = ic.kepler_orbit(1.0, 1.0, 1.0, 0.0)
        orbit = OracleOrbit(restatement, start, ic.kepler_period(1.0, 1.0, 1.0, 0.0) / steps,
                            integrator)
        orbit.step(steps)
        return max(math.dist((orbit.s["x"][i], orbit.s["y"][i], orbit.s["z"][i]),
                             (start["x"][i], start["y"][i], start["z"][i])) for i in range(2))

    order = closure_order(closure, COARSE[integrator])
    assert f"{order:.4f}" == PUBLISHED_ORDERS[integrator]


@pytest.mark.parametrize("integrator", ["vv", "yoshida4", "rk4"])
def test_the_oracle_holds_the_published_energy_envelopes(restatement, integrator):
    orbit = OracleOrbit(restatement, ic.kepler_orbit(1.0, 1.0, 1.0, 0.5),
                        ic.kepler_period(1.0, 1.0, 1.0, 0.5) / STEPS_PER_ORBIT, integrator)
    check_envelope(integrator, *envelope(orbit.step, orbit.energy))
