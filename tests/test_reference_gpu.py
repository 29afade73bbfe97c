"""Cross-checks against the reference's own CUDA solvers on the same device.

The reference's CudaDirectSolver and CudaTreeSolver (its .cu kernels built for
sm_100a by oracle/Makefile, target ref_cuda) run on the same inputs as this
backend: the tree's per-target accept decisions must give the same pair and
cell counts, and the forces must agree within the FP32 tolerances of each
path. Skipped where that library was not built.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import relative_errors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def reference_cuda():
    import oracle

    if not oracle.ReferenceCuda.built():
        pytest.skip("the reference's CUDA library (oracle/_ref) is not built here")
    ref = oracle.ReferenceCuda()
    if not ref.available():
        pytest.skip("the reference's CUDA solver finds no device")
    return ref


def test_direct_matches_the_reference_cuda_solver(b200, reference_cuda, golden_plummer):
    g = golden_plummer
    x, y, z, m = g["x"], g["y"], g["z"], g["m"]
    _, _, a_ref = reference_cuda.direct_timed(x, y, z, m, 0.01, repeats=1)
    exact = b200.B200DirectSolver(0.01, "fp64").evaluate((x, y, z), m)
    split = b200.B200DirectSolver(0.01, "split").evaluate((x, y, z), m)
    # The reference's CUDA kernel sums in FP64 in its own tile order.
    assert relative_errors(exact, a_ref).max() < 1e-12
    assert relative_errors(split, a_ref).max() < 2e-6


@pytest.mark.parametrize("n,quad", [(50_000, True), (200_000, False)])
def test_tree_counts_and_forces_match_the_reference_cuda_solver(b200, reference_cuda, n, quad):
    from orrery_b200 import initial_conditions as ic

    d = ic.galaxy_collision(n, softening=0.02, seed=20260821)
    x, y, z, m = (np.ascontiguousarray(d[k]) for k in ("x", "y", "z", "m"))
    _, _, a_ref, counts = reference_cuda.tree_timed(x, y, z, m, 0.02, 0.5, 32, quad, threads=4,
                                                     repeats=1)
    s = b200.B200TreeSolver(0.02, 0.5, 32, quad)
    a = s.evaluate((x, y, z), m)
    c = s.interaction_count()
    assert (c.particle_particle, c.particle_cell) == counts
    err = relative_errors(a, a_ref)
    assert err.max() < 1e-4 and np.sqrt(np.mean(err ** 2)) < 1e-5
