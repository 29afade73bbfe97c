"""Shared fixtures. Tests marked ``gpu`` need a B200; everything else runs on CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def restatement():
    """The oracle's C restatement of the reference path (built on demand)."""
    import oracle

    if not os.path.exists(oracle.RESTATEMENT_PATH):
        oracle.build(with_reference=False)
    return oracle.Restatement()


@pytest.fixture(scope="session")
def reference():
    """The reference's own CPU code; skipped where it was not built."""
    import oracle

    if not oracle.Reference.available():
        try:
            oracle.build()
        except Exception:  # noqa: BLE001 - sources absent on this machine
            pass
    if not oracle.Reference.available():
        pytest.skip("the reference library (oracle/_ref) is not built here")
    return oracle.Reference()


@pytest.fixture(scope="session")
def golden_plummer():
    return dict(np.load(os.path.join(GOLDEN, "plummer_2048.npz")))


@pytest.fixture(scope="session")
def golden_trajectory():
    return dict(np.load(os.path.join(GOLDEN, "trajectory_512.npz")))


@pytest.fixture(scope="session")
def b200():
    """The orrery_b200 package with its CUDA library loaded and a device present.

    Fails (never skips) when the library or the device is missing: a GPU test
    must not pass on a silent fallback."""
    import orrery_b200

    orrery_b200.load_library()
    assert orrery_b200.device_count() > 0, "no CUDA device visible to a gpu-marked test"
    return orrery_b200


def relative_errors(measured, exact):
    """Per-particle |a - a_ref| / |a_ref| for (N, 3) arrays."""
    measured = np.asarray(measured)
    exact = np.asarray(exact)
    mag = np.linalg.norm(exact, axis=1)
    diff = np.linalg.norm(measured - exact, axis=1)
    ok = mag > 0
    return diff[ok] / mag[ok]
