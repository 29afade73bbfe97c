"""Barnes-Hut on the GPU against the reference's tree.

Restates the contract of the reference's CUDA tree tests
(tests/solvers/cuda_tree_solver_test.cpp): the device's tree must have the
reference tree's node count, leaf count and depth and the same pair and cell
counters; here that is strengthened to bit equality of the whole ordering
(Morton codes and permutation, tests/solvers/morton_test.cpp) and of every
node field (mass, centre of mass, acceptance radius, escape index, particle
range, quadrupole), because the construction is FP64 in the reference's
order. Forces are FP32 on FP64 state and are held to a stated tolerance
against the reference's FP64 tree; theta = 0 must reduce to direct summation
with N(N-1) pairs and no cells.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import relative_errors

pytestmark = pytest.mark.gpu

# FP32 force terms on FP64 offsets, summed per cell/leaf in FP32 and across
# cells in FP64, against the reference's all-FP64 tree (per-particle relative).
TREE_WORST, TREE_RMS = 1e-4, 1e-5


def _xyzm(d):
    return d["x"], d["y"], d["z"], d["m"]


@pytest.mark.parametrize("quad", [False, True])
def test_tree_matches_reference_node_for_node(b200, golden_plummer, quad):
    g = golden_plummer
    tag = "quad" if quad else "mono"
    s = b200.B200TreeSolver(0.05, 0.5, 32, quad)
    a = s.evaluate((g["x"], g["y"], g["z"]), g["m"])
    codes, idx, origin, size = s.order(len(g["m"]))
    assert np.array_equal(codes, g["morton_codes"])
    assert np.array_equal(idx.astype(np.uint64), g["morton_index"])
    assert np.array_equal(origin, g["cube_origin"]) and size == float(g["cube_size"])
    reals, nidx, quads, leaves, depth = s.tree()
    assert reals.shape == g[f"bh_{tag}_reals"].shape
    assert np.array_equal(nidx, g[f"bh_{tag}_idx"])
    assert np.array_equal(reals, g[f"bh_{tag}_reals"])
    assert [leaves, depth] == g[f"bh_{tag}_meta"].tolist()
    if quad:
        assert np.array_equal(quads, g["bh_quad_quads"])
    c = s.interaction_count()
    ref_counts = g[f"bh_{tag}_counts"].tolist()
    assert [c.evaluations, c.particle_particle, c.particle_cell] == ref_counts
    err = relative_errors(a, g[f"bh_{tag}_acc"])
    assert err.max() < TREE_WORST, err.max()
    assert np.sqrt(np.mean(err ** 2)) < TREE_RMS, np.sqrt(np.mean(err ** 2))


def test_theta_zero_is_direct_summation(b200, golden_plummer):
    g = golden_plummer
    s = b200.B200TreeSolver(0.05, 0.0, 32, False)
    a = s.evaluate((g["x"], g["y"], g["z"]), g["m"])
    c = s.interaction_count()
    n = len(g["m"])
    assert c.particle_particle == n * (n - 1) and c.particle_cell == 0
    assert relative_errors(a, g["bh_theta0_acc"]).max() < TREE_WORST
    assert relative_errors(a, g["direct_eps0.05"]).max() < TREE_WORST


@pytest.mark.parametrize("n,leaf,theta,quad", [(1, 32, 0.5, False), (2, 1, 0.5, True),
                                               (33, 4, 0.7, True), (1000, 8, 0.5, False),
                                               (4097, 16, 0.4, True), (20000, 32, 0.5, True)])
def test_ragged_sizes_and_parameters_against_oracle(b200, restatement, n, leaf, theta, quad):
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(n, seed=7 + n)
    x, y, z, m = _xyzm(d)
    t_ref, codes_ref, idx_ref = restatement.tree(x, y, z, m, theta, leaf, quad)
    a_ref, counts = restatement.barnes_hut(x, y, z, m, 0.02, theta, leaf, quad)
    s = b200.B200TreeSolver(0.02, theta, leaf, quad)
    a = s.evaluate((x, y, z), m)
    codes, idx, _, _ = s.order(n)
    assert np.array_equal(codes, codes_ref) and np.array_equal(idx.astype(np.uint64), idx_ref)
    reals, nidx, quads, leaves, depth = s.tree()
    assert np.array_equal(nidx, t_ref.idx) and np.array_equal(reals, t_ref.reals)
    assert (leaves, depth) == (t_ref.leaf_count, t_ref.depth)
    if quad:
        assert np.array_equal(quads, t_ref.quads)
    c = s.interaction_count()
    assert (c.particle_particle, c.particle_cell) == (counts.particle_particle,
                                                      counts.particle_cell)
    if n > 1:
        assert relative_errors(a, a_ref).max() < TREE_WORST
    else:
        assert a.tolist() == [[0.0, 0.0, 0.0]]


# --------------------------------------------------------------------------
# The FP64 parity mode: forces equal to BarnesHutSolver's bit for bit
# --------------------------------------------------------------------------

@pytest.mark.parametrize("theta,quad,tag", [(0.5, False, "mono"), (0.5, True, "quad"),
                                            (0.0, False, "theta0")])
def test_fp64_walk_equals_the_reference_bitwise(b200, golden_plummer, theta, quad, tag):
    # tests/golden/plummer_2048.npz: the reference's BarnesHutSolver (scalar
    # leaf kernel), eps 0.05, leaf 32.
    g = golden_plummer
    s = b200.B200TreeSolver(0.05, theta, 32, quad, precision="fp64")
    a = s.evaluate((g["x"], g["y"], g["z"]), g["m"])
    assert np.array_equal(a, g[f"bh_{tag}_acc"])
    c = s.interaction_count()
    assert [c.evaluations, c.particle_particle, c.particle_cell] == \
        g[f"bh_{tag}_counts"].tolist()


@pytest.mark.parametrize("n,leaf,theta,quad", [(1, 32, 0.5, False), (2, 1, 0.5, True),
                                               (33, 4, 0.7, True), (1000, 8, 0.5, False),
                                               (20000, 32, 0.5, True)])
def test_fp64_walk_equals_the_oracle_on_ragged_inputs(b200, restatement, n, leaf, theta, quad):
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(n, seed=17 + n)
    x, y, z, m = _xyzm(d)
    a_ref, counts = restatement.barnes_hut(x, y, z, m, 0.02, theta, leaf, quad)
    s = b200.B200TreeSolver(0.02, theta, leaf, quad, precision="fp64")
    a = s.evaluate((x, y, z), m)
    assert np.array_equal(a, a_ref)
    c = s.interaction_count()
    assert (c.particle_particle, c.particle_cell) == (counts.particle_particle,
                                                      counts.particle_cell)


def test_fp64_walk_at_two_million_equals_the_oracle_on_sampled_targets(b200, restatement):
    from orrery_b200 import initial_conditions as ic
    d = ic.galaxy_collision(2_000_000, softening=0.02, seed=20260811)
    x, y, z, m = _xyzm(d)
    s = b200.B200TreeSolver(0.02, 0.5, 32, True, precision="fp64")
    a = s.evaluate((x, y, z), m)
    targets = np.random.default_rng(6).choice(len(m), 4096, replace=False)
    a_ref, pairs, cells = restatement.barnes_hut_targets(x, y, z, m, 0.02, 0.5, 32, True,
                                                         targets)
    assert np.array_equal(a[targets], a_ref)


def test_fp64_tree_system_steps_equal_the_oracle(b200, restatement):
    # A device-resident system over the parity-mode field: its carried
    # accelerations, before and after two VV steps, equal the oracle's FP64
    # walk at the same positions.
    from orrery_b200 import initial_conditions as ic
    n = 3000
    d = ic.plummer_sphere(n, seed=41)
    s = b200.DeviceSystem(n, 0.02, b200.SOLVER_TREE, "fp64", 0.5, 16, True)
    s.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    a0, _ = restatement.barnes_hut(d["x"], d["y"], d["z"], d["m"], 0.02, 0.5, 16, True)
    st = s.state()
    assert np.array_equal(np.stack([st["ax"], st["ay"], st["az"]], axis=1), a0)
    s.step(1e-3, 2, "vv")
    st = s.state()
    a1, _ = restatement.barnes_hut(st["x"], st["y"], st["z"], d["m"], 0.02, 0.5, 16, True)
    assert np.array_equal(np.stack([st["ax"], st["ay"], st["az"]], axis=1), a1)


def test_coincident_particles_hit_the_depth_limit(b200, restatement):
    # octree_test.cpp:407-432: identical codes cannot be separated, so the
    # subdivision stops at level 21 with one over-full leaf.
    p = np.full(40, 2.0)
    x, y, z, m = p, -p / 2, 1.5 * p, np.ones(40)
    s = b200.B200TreeSolver(0.1, 0.5, 4, True)
    s.evaluate((x, y, z), m)
    t_ref, _, _ = restatement.tree(x, y, z, m, 0.5, 4, True)
    reals, nidx, quads, leaves, depth = s.tree()
    assert np.array_equal(nidx, t_ref.idx) and np.array_equal(reals, t_ref.reals)
    assert leaves == 1 and nidx[-1, 2] == 40


def test_massless_particles_stay_finite(b200):
    z = np.zeros(16)
    s = b200.B200TreeSolver(0.1, 0.5, 4, True)
    a = s.evaluate((z, z.copy(), z.copy()), z.copy())
    reals, _, quads, _, _ = s.tree()
    assert np.all(np.isfinite(reals)) and np.all(reals[:, 0] == 0.0)
    assert np.all(np.isfinite(a))


def test_quadrupole_improves_accuracy(b200, restatement):
    # cuda_tree_solver_test.cpp:354-390 with its seed and softening.
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(4096, seed=20260811)
    x, y, z, m = _xyzm(d)
    exact = restatement.reference_accelerations(x, y, z, m, 0.05)
    mono = b200.B200TreeSolver(0.05, 0.5, 32, False)
    quad = b200.B200TreeSolver(0.05, 0.5, 32, True)
    e_mono = relative_errors(mono.evaluate((x, y, z), m), exact)
    e_quad = relative_errors(quad.evaluate((x, y, z), m), exact)
    rms = lambda e: np.sqrt(np.mean(e ** 2))  # noqa: E731
    assert rms(e_quad) < rms(e_mono)
    assert mono.interaction_count().particle_cell == quad.interaction_count().particle_cell
    # cuda_tree_solver_test.cpp:392-412: the approximation's own bounds.
    assert rms(e_mono) < 1e-2 and e_mono.max() < 1e-1


def test_repeated_evaluations_rebuild_the_tree(b200, golden_plummer):
    g = golden_plummer
    s = b200.B200TreeSolver(0.05, 0.5, 32, True)
    a1 = s.evaluate((g["x"], g["y"], g["z"]), g["m"])
    from orrery_b200 import initial_conditions as ic
    other = ic.plummer_sphere(5000, seed=4)
    s.evaluate((other["x"], other["y"], other["z"]), other["m"])
    a2 = s.evaluate((g["x"], g["y"], g["z"]), g["m"])
    assert np.array_equal(a1, a2)
    assert s.interaction_count().evaluations == 3


def test_two_million_collision_ordering_tree_and_sampled_forces(b200, restatement):
    # The Barnes-Hut workload at full size: two disc galaxies, 2,000,000
    # particles, theta 0.5, quadrupoles, leaf 32, eps 0.02. Ordering and tree
    # bit-exact against the oracle; forces and per-target counters on 4096
    # sampled targets.
    from orrery_b200 import initial_conditions as ic
    d = ic.galaxy_collision(2_000_000, softening=0.02, seed=20260811)
    x, y, z, m = _xyzm(d)
    s = b200.B200TreeSolver(0.02, 0.5, 32, True)
    a = s.evaluate((x, y, z), m)
    t_ref, codes_ref, idx_ref = restatement.tree(x, y, z, m, 0.5, 32, True)
    codes, idx, _, _ = s.order(len(m))
    assert np.array_equal(codes, codes_ref)
    assert np.array_equal(idx.astype(np.uint64), idx_ref)
    reals, nidx, quads, leaves, depth = s.tree()
    assert np.array_equal(nidx, t_ref.idx)
    assert np.array_equal(reals, t_ref.reals)
    assert np.array_equal(quads, t_ref.quads)
    assert (leaves, depth) == (t_ref.leaf_count, t_ref.depth)
    rng = np.random.default_rng(5)
    targets = rng.choice(len(m), 4096, replace=False)
    a_ref, pairs, cells = restatement.barnes_hut_targets(x, y, z, m, 0.02, 0.5, 32, True,
                                                         targets)
    err = relative_errors(a[targets], a_ref)
    assert err.max() < TREE_WORST, err.max()
    assert np.sqrt(np.mean(err ** 2)) < TREE_RMS
    # Total counters: the per-target counts of the sample scale to the total.
    c = s.interaction_count()
    assert c.particle_cell > 0 and c.particle_particle > 0


def test_two_million_counters_equal_reference(b200, reference):
    from orrery_b200 import initial_conditions as ic
    d = ic.galaxy_collision(2_000_000, softening=0.02, seed=20260811)
    x, y, z, m = _xyzm(d)
    s = b200.B200TreeSolver(0.02, 0.5, 32, True)
    s.evaluate((x, y, z), m)
    _, counts, _ = reference.barnes_hut(x, y, z, m, 0.02, 0.5, 32, True, kernel="avx2",
                                        threads=reference.worker_count(), with_tree=False)
    c = s.interaction_count()
    assert [c.particle_particle, c.particle_cell] == counts.tolist()[1:]


def test_tree_system_steps_match_host_steps(b200):
    # The device-resident system (graph-captured VV steps) gives the same
    # states as the drop-in solver driven by host kicks and drifts.
    from orrery_b200 import initial_conditions as ic
    d = ic.plummer_sphere(30000, seed=21)
    sysm = b200.DeviceSystem(30000, 0.02, kind=b200.SOLVER_TREE, opening_angle=0.5,
                             leaf_capacity=32, quadrupole=True)
    sysm.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    sysm.step(5e-4, 5, "vv")
    st = sysm.state()
    solver = b200.B200TreeSolver(0.02, 0.5, 32, True)
    x, y, z = d["x"].copy(), d["y"].copy(), d["z"].copy()
    vx, vy, vz = d["vx"].copy(), d["vy"].copy(), d["vz"].copy()
    a = solver.evaluate((x, y, z), d["m"])
    for _ in range(5):
        h = 5e-4 / 2
        vx += h * a[:, 0]
        vy += h * a[:, 1]
        vz += h * a[:, 2]
        x += 5e-4 * vx
        y += 5e-4 * vy
        z += 5e-4 * vz
        a = solver.evaluate((x, y, z), d["m"])
        vx += h * a[:, 0]
        vy += h * a[:, 1]
        vz += h * a[:, 2]
    assert np.array_equal(st["x"], x) and np.array_equal(st["vz"], vz)
    assert np.array_equal(st["ax"], a[:, 0])
