"""Host-side pieces of the benchmark that need no GPU: the serving stream is
seeded and has the stated mix, job inputs are valid systems, and the traffic
and roofline constants scale with the work."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_serving_stream_is_seeded_and_mixed():
    a = bench.make_stream(20.0)
    b = bench.make_stream(20.0)
    assert a == b
    assert abs(len(a) / 20.0 - 20.0) < 3.0  # Poisson at 20 jobs/s
    direct = [j for j in a if j["kind"] == "direct"]
    tree = [j for j in a if j["kind"] == "tree"]
    assert 0.6 < len(direct) / len(a) < 0.8
    assert all(1000 <= j["n"] <= 64000 and 200 <= j["steps"] <= 2000 for j in direct)
    assert all(100_000 <= j["n"] <= 4_000_000 and 100 <= j["steps"] <= 500 for j in tree)
    assert all(x["t"] < y["t"] for x, y in zip(a, a[1:]))


def test_job_states_are_valid_systems():
    jobs = [dict(t=0.0, kind="direct", n=1500, steps=200, offset=12345),
            dict(t=0.1, kind="direct", n=65536, steps=200, offset=7)]
    states = bench.job_states(jobs)
    for job, st in zip(jobs, states):
        assert set(st) == {"x", "y", "z", "vx", "vy", "vz", "m"}
        assert all(len(v) == job["n"] and np.all(np.isfinite(v)) for v in st.values())
        assert abs(st["m"].sum() - 1.0) < 1e-12
        # A subset of distinct template particles.
        assert len(np.unique(st["x"])) == job["n"]


def test_traffic_scales_with_the_work():
    t = bench.TRAFFIC_BYTES
    assert t[("walk", "fp32")](2_000_000) == 4 * t[("walk", "fp32")](500_000)
    assert t[("direct", "split")](262_144) > t[("direct", "fp32")](262_144)
    assert abs(t[("batch", "split")](1.7416705824e10) - 258.9e6) < 1.0
