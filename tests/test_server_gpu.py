"""The serving loop on the GPU: continuous batching must not change results.

A job's final state is the same whether it ran alone or in a mix of direct
and tree jobs that joined and left the batch around it (the batched kernel's
work items for one system do not depend on the other members, and every tree
job has its own pipeline), and matches the single-system paths.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def _direct(n, seed):
    from orrery_b200 import initial_conditions as ic
    return ic.plummer_sphere(n, scale_radius=1.0, seed=seed)


def _tree(n, seed):
    from orrery_b200 import initial_conditions as ic
    return ic.galaxy_collision(n, softening=0.02, seed=seed)


def _server(b200):
    return b200.Server(hbm_budget_bytes=20 << 30, direct_pairs_cap=10**10, max_tree_jobs=2)


def test_results_are_identical_alone_and_in_the_mix(b200):
    jobs = [("direct", _direct(3000, 1), 12), ("direct", _direct(700, 2), 30),
            ("tree", _tree(60000, 3), 4), ("direct", _direct(9000, 4), 5),
            ("tree", _tree(20000, 5), 6), ("direct", _direct(1500, 6), 20)]

    def submit(server, kind, state, steps):
        if kind == "direct":
            return server.submit(state, steps=steps, dt=1e-3, softening=0.01)
        return server.submit(state, steps=steps, dt=5e-4, softening=0.02, kind="tree",
                             integrator="vv", quadrupole=True)

    mix = _server(b200)
    ids = [submit(mix, *job) for job in jobs]
    mixed = [mix.wait(i, timeout=300) for i in ids]
    stats = mix.stats()
    mix.close()
    assert stats["completed"] == len(jobs)
    for (kind, state, steps), (report, final) in zip(jobs, mixed):
        assert report["status"] == b200.JOB_DONE and report["steps_done"] == steps
        alone = _server(b200)
        r, s = alone.wait(submit(alone, kind, state, steps), timeout=300)
        alone.close()
        assert all(np.array_equal(final[k], s[k]) for k in KEYS), kind


def test_served_direct_job_tracks_the_precision_system(b200):
    d = _direct(4000, 11)
    server = _server(b200)
    report, final = server.wait(server.submit(d, steps=10, dt=1e-3, softening=0.01),
                                timeout=120)
    server.close()
    system = b200.DeviceSystem(4000, 0.01, precision="split")
    system.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    system.step(1e-3, 10, "yoshida4")
    st = system.state()
    assert np.max(np.abs(final["x"] - st["x"])) < 1e-9
    assert np.max(np.abs(final["vy"] - st["vy"])) < 1e-8


def test_served_tree_job_equals_the_device_system(b200):
    d = _tree(50000, 12)
    server = _server(b200)
    report, final = server.wait(server.submit(d, steps=5, dt=5e-4, softening=0.02, kind="tree",
                                              integrator="vv", quadrupole=True), timeout=120)
    server.close()
    system = b200.DeviceSystem(50000, 0.02, kind=b200.SOLVER_TREE, opening_angle=0.5,
                               leaf_capacity=32, quadrupole=True)
    system.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    system.step(5e-4, 5, "vv")
    st = system.state()
    assert all(np.array_equal(final[k], st[k]) for k in KEYS)
