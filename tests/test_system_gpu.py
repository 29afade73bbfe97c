"""Device-resident integration against the reference's integrators.

With the FP64 direct field the device kick/drift and force are bit-identical
to the reference's host VelocityVerlet / Yoshida4 over DirectSolver, so whole
trajectories are compared for equality (tests/golden/trajectory_512.npz holds
the reference's own output). The FP32 and split fields are compared through
energy behaviour, as the reference's integrator tests do
(tests/integrators/energy_behaviour_test.cpp, conservation_test.cpp).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def _system(b200, g, precision, eps=0.01):
    n = len(g["m"])
    s = b200.DeviceSystem(n, eps, precision=precision)
    s.set_state(g["start_x"], g["start_y"], g["start_z"], g["start_vx"], g["start_vy"],
                g["start_vz"], g["m"])
    return s


@pytest.mark.parametrize("integrator,steps,tag", [("vv", 20, "vv20"), ("yoshida4", 10, "y4_10")])
def test_fp64_trajectory_is_bit_identical(b200, golden_trajectory, integrator, steps, tag):
    g = golden_trajectory
    s = _system(b200, g, "fp64")
    # The reference carried its own starting accelerations; they equal ours.
    st = s.state()
    for k in ("ax", "ay", "az"):
        assert np.array_equal(st[k], g[f"start_{k}"])
    s.step(1e-3, steps, integrator)
    st = s.state()
    for k in KEYS:
        assert np.array_equal(st[k], g[f"{tag}_{k}"]), k
    c = s.interaction_count()
    per = 3 if integrator == "yoshida4" else 1
    assert c.evaluations == 1 + steps * per
    assert c.particle_particle == c.evaluations * 512 * 511


def test_steps_split_across_calls_equal_one_call(b200, golden_trajectory):
    g = golden_trajectory
    a = _system(b200, g, "fp64")
    a.step(1e-3, 20, "vv")
    b = _system(b200, g, "fp64")
    for _ in range(4):
        b.step_async(1e-3, 5, "vv")
    b.synchronize()
    sa, sb = a.state(), b.state()
    assert all(np.array_equal(sa[k], sb[k]) for k in KEYS)


def test_fp64_rk4_trajectory_is_bit_identical(b200, golden_trajectory):
    # tests/golden/trajectory_rk4_512.npz: the reference's RungeKutta4 over its
    # scalar DirectSolver, 10 steps of dt 1e-3 from the same start.
    import os
    from conftest import GOLDEN
    rk4 = dict(np.load(os.path.join(GOLDEN, "trajectory_rk4_512.npz")))
    s = _system(b200, golden_trajectory, "fp64")
    s.step(1e-3, 10, "rk4")
    st = s.state()
    for k in KEYS:
        assert np.array_equal(st[k], rk4[f"rk4_10_{k}"]), k
    c = s.interaction_count()
    assert c.evaluations == 1 + 10 * 4


def test_rk4_over_the_tree_follows_the_exact_field(b200, golden_trajectory):
    # Barnes-Hut forces (theta 0.5, quadrupoles) carry ~1e-3 relative errors;
    # over five RK4 steps of 1e-3 they move positions by far less than 1e-6.
    g = golden_trajectory
    n = len(g["m"])
    t = b200.DeviceSystem(n, 0.01, b200.SOLVER_TREE, "fp32", 0.5, 32, True)
    t.set_state(g["start_x"], g["start_y"], g["start_z"], g["start_vx"], g["start_vy"],
                g["start_vz"], g["m"])
    e = _system(b200, g, "fp64")
    t.step(1e-3, 5, "rk4")
    e.step(1e-3, 5, "rk4")
    st, se = t.state(), e.state()
    for k in ("x", "y", "z"):
        assert np.max(np.abs(st[k] - se[k])) < 1e-6, k
    assert t.interaction_count().evaluations == 1 + 5 * 4


@pytest.mark.parametrize("integrator", ["vv", "yoshida4", "rk4"])
def test_host_state_steps_equal_resident_steps(b200, golden_trajectory, integrator):
    # Integrator::step over host arrays (upload, device step, download) is the
    # resident step: the carried accelerations make each call independent.
    g = golden_trajectory
    a = _system(b200, g, "fp64")
    a.step(1e-3, 3, integrator)
    b = _system(b200, g, "fp64")
    host = b.state()
    host["m"] = np.ascontiguousarray(g["m"], dtype=np.float64)
    for _ in range(3):
        b.step_host(host, 1e-3, 1, integrator)
    sa = a.state()
    assert all(np.array_equal(sa[k], host[k]) for k in KEYS)


def test_energies_are_bit_identical(b200, golden_plummer):
    g = golden_plummer
    s = b200.DeviceSystem(len(g["m"]), 0.01, precision="fp64")
    s.set_state(g["x"], g["y"], g["z"], g["vx"], g["vy"], g["vz"], g["m"])
    ke, pe = s.energy()
    assert pe == float(g["pe_eps0.01"])
    assert ke == float(g["ke"])


def test_c1_energy_and_forces_against_reference(b200, restatement):
    # Plummer N=4096, eps 0.01, velocity Verlet dt 1e-3, 100 steps: FP32 device
    # forces against the oracle's FP64 run of the same steps.
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(4096, seed=20260811)
    x, y, z, m = d["x"], d["y"], d["z"], d["m"]
    a0, _ = restatement.direct(x, y, z, m, 0.01)
    start = dict(x=x, y=y, z=z, vx=d["vx"], vy=d["vy"], vz=d["vz"], ax=a0[:, 0].copy(),
                 ay=a0[:, 1].copy(), az=a0[:, 2].copy())
    e0 = restatement.kinetic_energy(d["vx"], d["vy"], d["vz"], m) + \
        restatement.potential_energy(x, y, z, m, 0.01)
    ref, _ = restatement.integrate_direct(start, m, 0.01, 1e-3, 100, "vv")
    e_ref = restatement.kinetic_energy(ref["vx"], ref["vy"], ref["vz"], m) + \
        restatement.potential_energy(ref["x"], ref["y"], ref["z"], m, 0.01)
    for precision in ("fp32", "split"):
        s = b200.DeviceSystem(4096, 0.01, precision=precision)
        s.set_state(x, y, z, d["vx"], d["vy"], d["vz"], m)
        s.step(1e-3, 100, "vv")
        ke, pe = s.energy()
        drift_dev = (ke + pe - e0) / abs(e0)
        drift_ref = (e_ref - e0) / abs(e0)
        assert abs(drift_dev - drift_ref) < (1e-6 if precision == "fp32" else 1e-9), precision
        st = s.state()
        pos_err = np.max(np.abs(st["x"] - ref["x"]))
        assert pos_err < (1e-5 if precision == "fp32" else 1e-9), (precision, pos_err)


def test_momentum_conserved_over_steps(b200):
    # tests/integrators/conservation_test.cpp:94-123: 64 bodies, 200 steps,
    # dt 1e-3, eps 0.03; momentum to 64 * steps * machine epsilon * scale.
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(64, seed=9)
    s = b200.DeviceSystem(64, 0.03, precision="fp64")
    s.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    s.step(1e-3, 200, "vv")
    st = s.state()
    p = np.array([(st[k] * d["m"]).sum() for k in ("vx", "vy", "vz")])
    scale = (np.sqrt(st["vx"] ** 2 + st["vy"] ** 2 + st["vz"] ** 2) * d["m"]).sum()
    assert np.abs(p).max() <= 64 * 200 * np.finfo(float).eps * scale


def test_yoshida_energy_error_below_velocity_verlet(b200):
    # energy_behaviour_test.cpp:137-176: Yoshida-4's energy error is below VV's
    # at the same timestep.
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(1024, seed=11)
    errs = {}
    for integ in ("vv", "yoshida4"):
        s = b200.DeviceSystem(1024, 0.05, precision="fp64")
        s.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
        ke0, pe0 = s.energy()
        s.step(1e-2, 50, integ)
        ke, pe = s.energy()
        errs[integ] = abs((ke + pe) - (ke0 + pe0)) / abs(ke0 + pe0)
    assert errs["yoshida4"] < errs["vv"]


# -- the reference's integrator validation on Kepler orbits, on the device -----
# (tests/integrators/convergence_test.cpp, energy_behaviour_test.cpp; the
# figures are docs/validation.md's, which the oracle reproduces in
# tests/test_integrator_validation.py).

def _kepler_system(b200, orbit):
    s = b200.DeviceSystem(2, 0.0, precision="fp64")
    s.set_state(orbit["x"], orbit["y"], orbit["z"], orbit["vx"], orbit["vy"], orbit["vz"],
                orbit["m"])
    return s


@pytest.mark.parametrize("integrator", ["vv", "yoshida4", "rk4"])
def test_device_integrators_converge_at_the_published_orders(b200, integrator):
    import math

    from test_integrator_validation import COARSE, PUBLISHED_ORDERS, closure_order

    from orrery_b200 import initial_conditions as ic

    def closure(steps):
        start = ic.kepler_orbit(1.0, 1.0, 1.0, 0.0)
        s = _kepler_system(b200, start)
        s.step(ic.kepler_period(1.0, 1.0, 1.0, 0.0) / steps, steps, integrator)
        end = s.snapshot()
        return max(math.dist((end["x"][i], end["y"][i], end["z"][i]),
                             (start["x"][i], start["y"][i], start["z"][i])) for i in range(2))

    assert f"{closure_order(closure, COARSE[integrator]):.4f}" == PUBLISHED_ORDERS[integrator]


@pytest.mark.parametrize("integrator", ["vv", "yoshida4", "rk4"])
def test_device_integrators_hold_the_published_energy_envelopes(b200, integrator):
    from test_integrator_validation import STEPS_PER_ORBIT, check_envelope, envelope

    from orrery_b200 import initial_conditions as ic

    s = _kepler_system(b200, ic.kepler_orbit(1.0, 1.0, 1.0, 0.5))
    dt = ic.kepler_period(1.0, 1.0, 1.0, 0.5) / STEPS_PER_ORBIT

    def energy():
        d = s.diagnostics()
        return d["kinetic_energy"] + d["potential_energy"]

    check_envelope(integrator, *envelope(lambda k: s.step(dt, k, integrator), energy))


def test_the_device_orbit_takes_keplers_period(b200):
    # convergence_test.cpp: Yoshida-4 at 2000 steps an orbit; the period read
    # from the upward crossing of the separation's y component, within 1e-4
    # of Kepler's third law.
    from orrery_b200 import initial_conditions as ic

    params = (2.0, 1.0, 1.5, 0.5)
    expected = ic.kepler_period(*params)
    s = _kepler_system(b200, ic.kepler_orbit(*params))
    dt = expected / 2000
    measured = 0.0
    y = s.snapshot()["y"]
    previous = y[1] - y[0]
    for step in range(1, 4001):
        s.step(dt, 1, "yoshida4")
        y = s.snapshot()["y"]
        current = y[1] - y[0]
        if previous < 0 <= current:
            measured = (step - 1 + (-previous / (current - previous))) * dt
            break
        previous = current
    assert measured > 0 and abs(measured - expected) <= expected / 10000


@pytest.mark.parametrize("integrator", ["vv", "yoshida4", "rk4"])
def test_device_integrators_conserve_momenta_as_the_reference_requires(b200, reference,
                                                                        integrator):
    # conservation_test.cpp: 64 particles of the reference's Plummer sampler
    # (seed 20260810), softening 0.03, 200 steps of 0.001. Linear momentum
    # holds to round-off for every method; angular momentum to round-off for
    # the symmetric ones and to 1e-3 of itself for RK4.
    eps = float(np.finfo(np.float64).eps)

    def drift(a, b):
        return float(np.linalg.norm(np.asarray(b) - np.asarray(a)))

    d = reference.plummer(64, seed=20260810)
    s = b200.DeviceSystem(64, 0.03, precision="fp64")
    s.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    before = s.diagnostics()
    s.step(0.001, 200, integrator)
    after = s.diagnostics()
    bound = 64 * 200 * eps  # round_off_bound, times each quantity's scale
    linear_scale = np.sqrt(2 * before["kinetic_energy"])
    assert drift(before["linear_momentum"], after["linear_momentum"]) <= bound * linear_scale
    angular_scale = float(np.linalg.norm(before["angular_momentum"]))
    angular = drift(before["angular_momentum"], after["angular_momentum"])
    if integrator == "rk4":
        assert angular <= angular_scale / 1000
    else:
        assert angular <= bound * angular_scale


@pytest.mark.parametrize("integrator", ["vv", "yoshida4", "rk4"])
def test_a_step_leaves_the_accelerations_agreeing_with_the_positions(b200, integrator):
    # integrator_test.cpp: after two steps of 0.01 on a Kepler orbit (masses 2
    # and 1, a = 1, e = 0.3) the carried accelerations are exactly those a
    # fresh evaluation of the positions gives.
    from orrery_b200 import initial_conditions as ic

    orbit = ic.kepler_orbit(2.0, 1.0, 1.0, 0.3)
    s = _kepler_system(b200, orbit)
    s.step(0.01, 2, integrator)
    st = s.state()
    fresh = b200.B200DirectSolver(0.0, "fp64").evaluate((st["x"], st["y"], st["z"]), orbit["m"])
    assert np.array_equal(np.stack([st["ax"], st["ay"], st["az"]], axis=1), fresh)


@pytest.mark.parametrize("integrator", ["vv", "yoshida4"])
def test_the_symmetric_methods_run_backwards_to_where_they_started(b200, integrator):
    # integrator_test.cpp: 200 steps of 0.002 and 200 of -0.002 on a Kepler
    # orbit (masses 3 and 1, a = 1, e = 0.4, softening 0.01) return positions
    # and velocities to within 64 * 200 machine epsilons.
    from orrery_b200 import initial_conditions as ic

    start = ic.kepler_orbit(3.0, 1.0, 1.0, 0.4)
    s = b200.DeviceSystem(2, 0.01, precision="fp64")
    s.set_state(start["x"], start["y"], start["z"], start["vx"], start["vy"], start["vz"],
                start["m"])
    s.step(0.002, 200, integrator)
    s.step(-0.002, 200, integrator)
    end = s.state()
    tolerance = 64 * 200 * float(np.finfo(np.float64).eps)
    for i in range(2):
        for keys in (("x", "y", "z"), ("vx", "vy", "vz")):
            error = np.linalg.norm([end[k][i] - start[k][i] for k in keys])
            assert error <= tolerance, (i, keys, error)
