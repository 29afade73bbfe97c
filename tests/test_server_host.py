"""The serving loop's scheduler on the CPU (fake-device mode: no GPU, each
step takes the time the cost model gives). Failures are made on the host:
jobs that can never fit are refused, cancelled jobs leave the queue, a full
budget holds jobs back, malformed specs are errors.
"""
from __future__ import annotations

import numpy as np
import pytest

import orrery_b200 as ob


def _state(n, seed=0):
    rng = np.random.default_rng(seed)
    return {"x": rng.normal(size=n), "y": rng.normal(size=n), "z": rng.normal(size=n),
            "vx": np.zeros(n), "vy": np.zeros(n), "vz": np.zeros(n), "m": np.full(n, 1.0 / n)}


@pytest.fixture
def server():
    s = ob.Server(hbm_budget_bytes=1 << 34, direct_pairs_cap=10**9, max_tree_jobs=1, fake=True,
                  fake_direct_gint_s=100.0, fake_tree_ns_per_particle=50.0)
    yield s
    s.close()


def test_jobs_complete_and_return_their_state(server):
    a = server.submit(_state(1000, 1), steps=20, dt=1e-3, softening=0.01)
    b = server.submit(_state(50000, 2), steps=3, dt=5e-4, softening=0.02, kind="tree",
                      integrator="vv")
    ra, sa = server.wait(a, timeout=30)
    rb, sb = server.wait(b, timeout=30)
    assert ra["status"] == ob.JOB_DONE and ra["steps_done"] == 20
    assert rb["status"] == ob.JOB_DONE and rb["steps_done"] == 3
    assert np.array_equal(sa["x"], _state(1000, 1)["x"])  # fake mode returns the input
    st = server.stats()
    assert st["completed"] == 2 and st["running"] == 0 and st["queued"] == 0
    assert st["job_latency_p99_s"] >= st["job_latency_p50_s"] > 0
    assert st["step_latency_p50_ms"] > 0


def test_a_job_is_submitted_as_the_references_particle_data(server):
    # The reference's make_initial_conditions gives a ParticleData
    # (position_x ... mass); it is submitted as it is.
    from types import SimpleNamespace

    st = _state(800, 3)
    data = SimpleNamespace(position_x=st["x"], position_y=st["y"], position_z=st["z"],
                           velocity_x=st["vx"], velocity_y=st["vy"], velocity_z=st["vz"],
                           mass=st["m"])
    report, final = server.wait(server.submit(data, steps=4, dt=1e-3, softening=0.01),
                                timeout=30)
    assert report["status"] == ob.JOB_DONE and report["steps_done"] == 4
    assert np.array_equal(final["y"], st["y"])  # fake mode returns the input


def test_direct_jobs_share_batched_steps(server):
    # Eight direct jobs submitted together step together: all finish after
    # about the time of their 10 shared steps, not 8 x 10 separate ones.
    ids = [server.submit(_state(2000, k), steps=10, dt=1e-3, softening=0.01) for k in range(8)]
    reports = [server.wait(i, timeout=30, outputs=False)[0] for i in ids]
    assert all(r["status"] == ob.JOB_DONE for r in reports)
    admitted = [r["admitted_s"] for r in reports]
    assert max(admitted) - min(admitted) < 0.05


def test_tree_jobs_respect_their_concurrency_cap(server):
    ids = [server.submit(_state(200000, k), steps=2, dt=5e-4, softening=0.02, kind="tree",
                         integrator="vv") for k in range(3)]
    reports = sorted((server.wait(i, timeout=60, outputs=False)[0] for i in ids),
                     key=lambda r: r["admitted_s"])
    # max_tree_jobs = 1: each starts after the previous one finished (FIFO).
    for before, after in zip(reports, reports[1:]):
        assert after["admitted_s"] >= before["finished_s"] - 1e-3
    assert [r["id"] for r in reports] == ids


def test_budget_holds_jobs_back_until_memory_frees():
    # A budget that fits one 100k-particle tree job at a time.
    s = ob.Server(hbm_budget_bytes=60_000_000, max_tree_jobs=4, fake=True,
                  fake_direct_gint_s=100.0, fake_tree_ns_per_particle=100.0)
    try:
        ids = [s.submit(_state(100000, k), steps=2, dt=5e-4, softening=0.02, kind="tree",
                        integrator="vv") for k in range(3)]
        reports = [s.wait(i, timeout=60, outputs=False)[0] for i in ids]
        reports.sort(key=lambda r: r["admitted_s"])
        for before, after in zip(reports, reports[1:]):
            assert after["admitted_s"] >= before["finished_s"] - 1e-3
        assert s.stats()["hbm_peak"] <= 60_000_000
    finally:
        s.close()


def test_a_job_that_never_fits_is_refused():
    s = ob.Server(hbm_budget_bytes=10_000_000, fake=True)
    try:
        with pytest.raises(ob.OrreryError) as err:
            s.submit(_state(1_000_000), steps=1, dt=1e-3, softening=0.01, kind="tree")
        assert err.value.code == ob.ERROR_CAPACITY
        assert s.stats()["rejected"] == 1
    finally:
        s.close()


def test_direct_work_cap_is_respected():
    s = ob.Server(hbm_budget_bytes=1 << 34, direct_pairs_cap=2 * 3000 * 2999, fake=True,
                  fake_direct_gint_s=1.0)
    try:
        ids = [s.submit(_state(3000, k), steps=5, dt=1e-3, softening=0.01) for k in range(4)]
        reports = [s.wait(i, timeout=60, outputs=False)[0] for i in ids]
        # Two run together, the next two wait for them.
        assert reports[2]["admitted_s"] >= min(reports[0]["finished_s"],
                                               reports[1]["finished_s"]) - 1e-3
        with pytest.raises(ob.OrreryError):
            s.submit(_state(5000), steps=1, dt=1e-3, softening=0.01)  # above the cap alone
    finally:
        s.close()


def test_work_units_are_the_reference_cost_model():
    # tests/golden/work_units.json: service/orrery_service/limits.py's own
    # work_units, written by tests/golden/make_golden_work_units.py.
    import json
    import os
    from conftest import GOLDEN
    with open(os.path.join(GOLDEN, "work_units.json")) as fh:
        g = json.load(fh)
    for case in g["cases"]:
        assert ob.work_units(case["count"], case["steps"], case["solver"]) == case["work"], case
    assert ob.work_units(g["MAX_PARTICLES"], 6000, "barnes-hut") == g["MAX_WORK"]


def test_a_job_above_the_work_ceiling_is_refused():
    ceiling = ob.work_units(1000, 20, "direct")
    s = ob.Server(hbm_budget_bytes=1 << 34, fake=True, max_job_work=ceiling)
    try:
        ok = s.submit(_state(1000), steps=20, dt=1e-3, softening=0.01)
        with pytest.raises(ob.OrreryError) as err:
            s.submit(_state(1000), steps=21, dt=1e-3, softening=0.01)
        assert err.value.code == ob.ERROR_CAPACITY
        assert s.wait(ok, timeout=60, outputs=False)[0]["status"] == ob.JOB_DONE
        assert s.stats()["rejected"] == 1
    finally:
        s.close()


def test_running_work_holds_jobs_back():
    # Three equal direct jobs under a cap of one and a half jobs' work: they run
    # one after another (a job alone always runs).
    w = ob.work_units(3000, 5, "direct")
    s = ob.Server(hbm_budget_bytes=1 << 34, fake=True, fake_direct_gint_s=1.0,
                  max_running_work=1.5 * w)
    try:
        ids = [s.submit(_state(3000, k), steps=5, dt=1e-3, softening=0.01) for k in range(3)]
        r = [s.wait(i, timeout=60, outputs=False)[0] for i in ids]
        assert r[1]["admitted_s"] >= r[0]["finished_s"] - 1e-3
        assert r[2]["admitted_s"] >= r[1]["finished_s"] - 1e-3
        big = s.submit(_state(6000), steps=5, dt=1e-3, softening=0.01)  # above the cap alone
        assert s.wait(big, timeout=60, outputs=False)[0]["status"] == ob.JOB_DONE
    finally:
        s.close()


def test_cancelled_jobs_stop(server):
    slow = ob.Server(hbm_budget_bytes=1 << 34, max_tree_jobs=1, fake=True,
                     fake_tree_ns_per_particle=1000.0)
    try:
        first = slow.submit(_state(100000, 1), steps=50, dt=5e-4, softening=0.02, kind="tree")
        queued = slow.submit(_state(100000, 2), steps=50, dt=5e-4, softening=0.02, kind="tree")
        slow.cancel(queued)
        slow.cancel(first)
        r1, _ = slow.wait(first, timeout=30, outputs=False)
        r2, _ = slow.wait(queued, timeout=30, outputs=False)
        assert r1["status"] == ob.JOB_CANCELLED and r2["status"] == ob.JOB_CANCELLED
        assert r1["steps_done"] < 50
        slow.drain(timeout=10)
        assert slow.stats()["cancelled"] == 2
    finally:
        slow.close()


def test_malformed_specs_are_errors(server):
    with pytest.raises(ob.OrreryError):
        server.submit(_state(100), steps=0, dt=1e-3, softening=0.01)
    with pytest.raises(ob.OrreryError):
        server.submit(_state(100), steps=5, dt=float("nan"), softening=0.01)
    with pytest.raises(ob.OrreryError):
        server.submit(_state(100), steps=5, dt=1e-3, softening=0.0)  # direct needs eps > 0
    with pytest.raises(ob.OrreryError):
        server.wait(987654, timeout=0.1)


def test_wait_times_out_while_a_job_runs():
    s = ob.Server(hbm_budget_bytes=1 << 34, fake=True, fake_tree_ns_per_particle=2000.0)
    try:
        j = s.submit(_state(200000), steps=100, dt=5e-4, softening=0.02, kind="tree")
        with pytest.raises(ob.OrreryError) as err:
            s.wait(j, timeout=0.05)
        assert err.value.code == ob.ERROR_TIMEOUT
        s.cancel(j)
        s.wait(j, timeout=30, outputs=False)
    finally:
        s.close()


def test_any_timeout_is_a_deadline_the_clock_can_hold():
    # An infinite wait must not overflow the deadline's conversion to clock
    # ticks; NaN or a negative timeout waits not at all.
    s = ob.Server(hbm_budget_bytes=1 << 34, direct_pairs_cap=10**9, max_tree_jobs=1, fake=True,
                  fake_direct_gint_s=100.0, fake_tree_ns_per_particle=50.0)
    try:
        slow = s.submit(_state(3000, 5), steps=2000, dt=1e-3, softening=0.01)  # ~0.2 s modelled
        for timeout in (float("nan"), -1.0):
            with pytest.raises(ob.OrreryError) as e:
                s.wait(slow, timeout=timeout)
            assert e.value.code == ob.ERROR_TIMEOUT
        report, _ = s.wait(slow, timeout=float("inf"))
        assert report["status"] == ob.JOB_DONE and report["steps_done"] == 2000
        s.drain(timeout=float("inf"))
    finally:
        s.close()


def test_an_unknown_job_kind_or_integrator_is_refused(server):
    # A misspelt kind must not quietly become a Barnes-Hut job.
    for kw in (dict(kind="drect"), dict(kind="barnes-hut"), dict(integrator="leapfrog")):
        with pytest.raises(ob.OrreryError) as e:
            server.submit(_state(100), steps=2, dt=1e-3, softening=0.01, **kw)
        assert e.value.code == ob.ERROR_INVALID_ARGUMENT
    assert server.stats()["queued"] == 0
