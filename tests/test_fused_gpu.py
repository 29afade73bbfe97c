"""Whole steps of a small FP32-direct system in one cooperative launch.

At a few thousand particles the fused path (`ob_system_set_fused_steps`)
replaces the four launches of each velocity-Verlet or Yoshida-4 substep with
one kernel. Its kicks and drifts are the same explicitly rounded FP64
operations as the separate kernels, and its forces are the FP32 direct
arithmetic with its own summation order, so the checks are: the forces it
carries stay within the FP32 direct kernel's bounds of the FP64 oracle (the
reference's FP32 CUDA bounds, worst < 2e-4, RMS < 2e-5); trajectories stay
beside those of the separate kernels and of the FP64 oracle; steps split
across calls equal one call bit for bit; counters and energy behave.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import relative_errors

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def _plummer(n, seed=3):
    from orrery_b200 import initial_conditions as ic
    return ic.plummer_sphere(n, seed=seed)


def _system(b200, d, eps=0.01, fused=True):
    n = len(d["m"])
    s = b200.DeviceSystem(n, eps, precision="fp32")
    active = s.set_fused_steps(fused)
    s.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    return s, active


# 5500: more CTAs than SMs, so the launch takes the 16-warp kernel at two
# CTAs per SM; the others take the 32-warp kernel.
@pytest.mark.parametrize("n", [2, 33, 1000, 4096, 5500])
@pytest.mark.parametrize("integrator,steps", [("vv", 10), ("yoshida4", 4)])
def test_fused_steps_carry_forces_within_the_fp32_bounds(b200, restatement, n, integrator, steps):
    d = _plummer(n)
    s, active = _system(b200, d)
    assert active
    assert s.step_kernels(1e-3, integrator) == 1
    s.step(1e-3, steps, integrator)
    st = s.state()
    a = np.stack([st["ax"], st["ay"], st["az"]], axis=1)
    exact, _ = restatement.direct(st["x"], st["y"], st["z"], d["m"], 0.01)
    err = relative_errors(a, exact)
    assert err.max() < 2e-4 and np.sqrt(np.mean(err ** 2)) < 2e-5, (err.max(), err.mean())
    c = s.interaction_count()
    per = 3 if integrator == "yoshida4" else 1
    assert c.evaluations == 1 + steps * per
    assert c.particle_particle == c.evaluations * n * (n - 1)


def test_fused_trajectory_stays_beside_the_separate_kernels_and_the_oracle(b200, restatement):
    d = _plummer(4096, seed=21)
    fused, on = _system(b200, d)
    plain, off = _system(b200, d, fused=False)
    assert on and not off
    fused.step(1e-3, 50, "vv")
    plain.step(1e-3, 50, "vv")
    a0, _ = restatement.direct(d["x"], d["y"], d["z"], d["m"], 0.01)
    start = dict(x=d["x"], y=d["y"], z=d["z"], vx=d["vx"], vy=d["vy"], vz=d["vz"],
                 ax=a0[:, 0].copy(), ay=a0[:, 1].copy(), az=a0[:, 2].copy())
    ref, _ = restatement.integrate_direct(start, d["m"], 0.01, 1e-3, 50, "vv")
    f, p = fused.state(), plain.state()
    for k in ("x", "y", "z"):
        assert np.max(np.abs(f[k] - ref[k])) < 1e-5
        assert np.max(np.abs(f[k] - p[k])) < 1e-5
    ke, pe = fused.energy()
    ke0 = restatement.kinetic_energy(d["vx"], d["vy"], d["vz"], d["m"])
    pe0 = restatement.potential_energy(d["x"], d["y"], d["z"], d["m"], 0.01)
    assert abs((ke + pe) - (ke0 + pe0)) / abs(ke0 + pe0) < 1e-5


def test_fused_steps_split_across_calls_equal_one_call(b200):
    d = _plummer(3000, seed=8)
    a, _ = _system(b200, d)
    b, _ = _system(b200, d)
    a.step(1e-3, 12, "yoshida4")
    for _ in range(4):
        b.step_async(1e-3, 3, "yoshida4")
    b.synchronize()
    sa, sb = a.state(), b.state()
    assert all(np.array_equal(sa[k], sb[k]) for k in KEYS)


def test_fused_host_steps_equal_resident_steps(b200):
    # Integrator::step over host arrays (upload, one fused launch, download)
    # is the resident fused step, bit for bit.
    d = _plummer(2048, seed=9)
    a, on_a = _system(b200, d)
    b, on_b = _system(b200, d)
    assert on_a and on_b
    a.step(1e-3, 3, "vv")
    host = b.state()
    host["m"] = np.ascontiguousarray(d["m"], dtype=np.float64)
    for _ in range(3):
        b.step_host(host, 1e-3, 1, "vv")
    sa = a.state()
    assert all(np.array_equal(sa[k], host[k]) for k in KEYS)


def test_a_heavy_target_skips_itself(b200, restatement):
    # m / eps^3 above the FP32 range (1e30 / 1e-9): the target's own entry
    # must be skipped by index (0 * inf would otherwise poison its sum); its
    # neighbours, at least ~0.01 away, still see finite FP32 terms.
    d = _plummer(500, seed=4)
    m = d["m"].copy()
    m[7] = 1e30
    d = dict(d, m=m)
    s, active = _system(b200, d, eps=1e-3)
    assert active
    s.step(1e-6, 1, "vv")
    st = s.state()
    a = np.stack([st["ax"], st["ay"], st["az"]], axis=1)
    assert np.all(np.isfinite(a))
    exact, _ = restatement.direct(st["x"], st["y"], st["z"], m, 1e-3)
    err = relative_errors(a, exact)
    assert np.median(err) < 2e-5


def test_unsoftened_or_large_systems_use_the_separate_kernels(b200):
    assert not _system(b200, _plummer(64), eps=0.0)[1]
    assert not _system(b200, _plummer(60000))[1]
