"""Pins the oracle restatement (oracle/oracle.c) before any GPU result is
compared with it.

Three kinds of check:
  * the known-answer tests of the reference's own suites
    (tests/solvers/morton_test.cpp, octree_test.cpp, direct_solver_test.cpp,
    cuda_direct_solver_test.cpp), restated;
  * bit-for-bit agreement with the golden fixtures, which are outputs of the
    reference's compiled code (tests/golden/make_golden.py);
  * bit-for-bit agreement with the reference library itself on fresh seeds,
    where oracle/_ref is built.
"""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

from conftest import GOLDEN


# --------------------------------------------------------------------------
# Morton known answers (tests/solvers/morton_test.cpp:45-181)
# --------------------------------------------------------------------------

def test_spread_bits_known_answers(restatement):
    r = restatement
    assert r.spread_bits(0) == 0
    assert r.spread_bits(1) == 1
    assert r.spread_bits(2) == 0b1000
    assert r.spread_bits(3) == 0b1001
    assert r.spread_bits(0b101) == 0b1000001
    assert r.spread_bits(1 << 20) == 1 << 60
    for bit in range(21):
        assert r.spread_bits(1 << bit) == 1 << (3 * bit)
    assert r.spread_bits(1 << 21) == 0


def test_interleave_order(restatement):
    r = restatement
    assert r.morton_code_grid(0, 0, 0) == 0
    assert r.morton_code_grid(1, 0, 0) == 0b100
    assert r.morton_code_grid(0, 1, 0) == 0b010
    assert r.morton_code_grid(0, 0, 1) == 0b001
    assert r.morton_code_grid(1, 1, 1) == 0b111
    assert r.morton_code_grid(2, 0, 0) == 0b100000
    assert r.morton_code_grid(2, 1, 1) == 0b100011


def test_octant_of_code(restatement):
    r = restatement
    grid = 1 << 21
    corner = r.morton_code_grid(grid - 1, 0, grid - 1)
    for level in range(1, 22):
        assert r.morton_octant(corner, level) == 0b101
    single = r.morton_code_grid(1 << 18, 0, 0)
    assert [r.morton_octant(single, lv) for lv in (1, 2, 3, 4)] == [0, 0, 0b100, 0]
    assert r.morton_octant(corner, 0) == 0
    assert r.morton_octant(corner, 22) == 0


def test_bounding_cube_known_answer(restatement):
    x = np.array([-2.0, 4.0])
    y = np.array([0.0, 1.0])
    z = np.array([1.0, 3.0])
    origin, size = restatement.bounding_cube(x, y, z)
    assert size == 6.0
    centre = origin + size / 2
    assert list(centre) == [1.0, 0.5, 2.0]


def test_degenerate_and_empty_cubes(restatement):
    x = np.array([3.0, 3.0])
    origin, size = restatement.bounding_cube(x, x.copy(), x.copy())
    assert size > 0
    assert list(origin + size / 2) == [3.0, 3.0, 3.0]
    e = np.zeros(0)
    origin, size = restatement.bounding_cube(e, e, e)
    assert size == 0.0
    assert restatement.morton_code(np.zeros(3), origin, size) == 0


def test_far_face_clamp(restatement):
    grid = 1 << 21
    last = restatement.morton_code_grid(grid - 1, grid - 1, grid - 1)
    assert restatement.morton_code(np.ones(3), np.zeros(3), 1.0) == last
    assert restatement.morton_code(-np.ones(3), np.zeros(3), 1.0) == 0


def test_ordering_is_a_permutation_with_ascending_codes(restatement, golden_plummer):
    g = golden_plummer
    codes, idx, origin, size = restatement.morton_order(g["x"], g["y"], g["z"])
    assert np.array_equal(np.sort(idx), np.arange(len(idx), dtype=np.uint64))
    assert np.all(codes[1:] >= codes[:-1])
    ties = codes[1:] == codes[:-1]
    assert np.all(idx[1:][ties] > idx[:-1][ties])


# --------------------------------------------------------------------------
# Direct known answers (tests/solvers/direct_solver_test.cpp:93-260,
# cuda_direct_solver_test.cpp:296-337)
# --------------------------------------------------------------------------

def test_two_body_pair_is_exact(restatement):
    a, counts = restatement.direct(np.array([-1.0, 1.0]), np.zeros(2), np.zeros(2),
                                   np.array([2.0, 3.0]), 0.0)
    assert a[0].tolist() == [0.75, 0.0, 0.0]
    assert a[1].tolist() == [-0.5, 0.0, 0.0]
    assert counts.particle_particle == 2


def test_three_four_twelve(restatement):
    a, _ = restatement.direct(np.array([0.0, 3.0]), np.array([0.0, 4.0]),
                              np.array([0.0, 12.0]), np.array([1.0, 2.0]), 0.0)
    expected = np.array([3.0, 4.0, 12.0]) * (2.0 / 13.0 ** 3)
    assert np.linalg.norm(a[0] - expected) <= 8 * np.finfo(float).eps * np.linalg.norm(expected)


def test_plummer_softening_factor(restatement):
    a, _ = restatement.direct(np.array([0.0, 4.0]), np.zeros(2), np.zeros(2),
                              np.array([1.0, 5.0]), 3.0)
    expected = 5.0 * 4.0 / (16.0 + 9.0) ** 1.5
    assert abs(a[0, 0] - expected) <= 8 * np.finfo(float).eps * expected
    assert a[0, 1] == 0.0 and a[0, 2] == 0.0


def test_counts_for_five_particles(restatement):
    x = np.arange(5.0)
    _, counts = restatement.direct(x, x * 0, x * 0, np.ones(5), 0.1)
    assert counts.particle_particle == 20
    assert counts.evaluations == 1


def test_origin_particle_kat(restatement):
    a, _ = restatement.direct(np.array([0.0, 1.0, 0.0]), np.array([0.0, 0.0, 2.0]),
                              np.zeros(3), np.ones(3), 0.0)
    assert a[0].tolist() == [1.0, 0.25, 0.0]


def test_empty_and_single(restatement):
    a, counts = restatement.direct(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), 0.1)
    assert a.shape == (0, 3) and counts.particle_particle == 0
    a, counts = restatement.direct(np.ones(1), np.ones(1), np.ones(1), np.ones(1), 0.0)
    assert a.tolist() == [[0.0, 0.0, 0.0]] and counts.particle_particle == 0


# --------------------------------------------------------------------------
# Octree known answers (tests/solvers/octree_test.cpp:98-451)
# --------------------------------------------------------------------------

def test_single_leaf_known_answer(restatement):
    t, _, _ = restatement.tree(np.array([-1.0, 1.0]), np.zeros(2), np.zeros(2),
                               np.array([2.0, 3.0]), 0.5, 8)
    assert t.node_count == 1 and t.leaf_count == 1 and t.depth == 0
    assert t.idx[0].tolist() == [1, 0, 2]
    assert t.reals[0, 0] == 5.0
    assert t.reals[0, 1] == 1.0 / 5.0 and t.reals[0, 2] == 0.0 and t.reals[0, 3] == 0.0


def test_acceptance_radius_known_answer(restatement):
    t, _, _ = restatement.tree(np.array([-1.0, 1.0]), np.zeros(2), np.zeros(2),
                               np.array([3.0, 1.0]), 0.5, 8)
    expected = (2 / 0.5 + 0.5) ** 2
    assert abs(t.reals[0, 4] - expected) <= 8 * np.finfo(float).eps * 4 * expected


def test_theta_zero_accepts_nothing(restatement, golden_plummer):
    g = golden_plummer
    t, _, _ = restatement.tree(g["x"][:100], g["y"][:100], g["z"][:100], g["m"][:100], 0.0, 8)
    assert np.all(np.isinf(t.reals[:, 4]))


def test_depth_limit_with_coincident_particles(restatement):
    p = np.full(40, 2.0)
    t, _, _ = restatement.tree(p, -p / 2, 1.5 * p, np.ones(40), 0.5, 4)
    assert t.leaf_count == 1
    assert t.idx[-1, 2] == 40
    assert t.reals[-1, 0] == 40.0
    assert 0 < t.reals[-1, 4] < math.inf


def test_massless_particles_stay_finite(restatement):
    z = np.zeros(16)
    t, _, _ = restatement.tree(z, z.copy(), z.copy(), z.copy(), 0.5, 4, quadrupole=True)
    assert np.all(t.reals[:, 0] == 0.0)
    assert np.all(np.isfinite(t.reals))


def test_leaves_partition_and_escape_indices(restatement, golden_plummer):
    g = golden_plummer
    t, _, _ = restatement.tree(g["x"], g["y"], g["z"], g["m"], 0.5, 8)
    n = len(g["m"])
    seen = np.zeros(n, int)
    for k in range(t.node_count):
        nxt, first, count = (int(v) for v in t.idx[k])
        assert k < nxt <= t.node_count
        if count:
            assert nxt == k + 1 and count <= 8
            seen[first:first + count] += 1
    assert np.all(seen == 1)


# --------------------------------------------------------------------------
# Bit-for-bit against the reference's outputs (golden fixtures)
# --------------------------------------------------------------------------

def test_direct_matches_reference_bitwise(restatement, golden_plummer):
    g = golden_plummer
    for eps in (0.01, 0.05):
        a, counts = restatement.direct(g["x"], g["y"], g["z"], g["m"], eps)
        assert np.array_equal(a, g[f"direct_eps{eps}"])
        assert counts.particle_particle == int(g["direct_pairs"])


def test_morton_matches_reference_bitwise(restatement, golden_plummer):
    g = golden_plummer
    codes, idx, origin, size = restatement.morton_order(g["x"], g["y"], g["z"])
    assert np.array_equal(codes, g["morton_codes"])
    assert np.array_equal(idx, g["morton_index"])
    assert np.array_equal(origin, g["cube_origin"]) and size == float(g["cube_size"])


@pytest.mark.parametrize("quad", [False, True])
def test_tree_and_walk_match_reference_bitwise(restatement, golden_plummer, quad):
    g = golden_plummer
    tag = "quad" if quad else "mono"
    t, _, _ = restatement.tree(g["x"], g["y"], g["z"], g["m"], 0.5, 32, quad)
    assert np.array_equal(t.reals, g[f"bh_{tag}_reals"])
    assert np.array_equal(t.idx, g[f"bh_{tag}_idx"])
    assert [t.leaf_count, t.depth] == g[f"bh_{tag}_meta"].tolist()
    if quad:
        assert np.array_equal(t.quads, g["bh_quad_quads"])
    a, counts = restatement.barnes_hut(g["x"], g["y"], g["z"], g["m"], 0.05, 0.5, 32, quad)
    assert np.array_equal(a, g[f"bh_{tag}_acc"])
    assert [counts.evaluations, counts.particle_particle, counts.particle_cell] == \
        g[f"bh_{tag}_counts"].tolist()


def test_theta_zero_is_direct_summation(restatement, golden_plummer):
    g = golden_plummer
    a, counts = restatement.barnes_hut(g["x"], g["y"], g["z"], g["m"], 0.05, 0.0, 32, False)
    assert np.array_equal(a, g["bh_theta0_acc"])
    n = len(g["m"])
    assert counts.particle_particle == n * (n - 1) and counts.particle_cell == 0


@pytest.mark.parametrize("integrator,steps,tag", [("vv", 20, "vv20"), ("yoshida4", 10, "y4_10")])
def test_integrators_match_reference_bitwise(restatement, golden_trajectory, integrator, steps,
                                             tag):
    g = golden_trajectory
    keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
    state = {k: g[f"start_{k}"] for k in keys}
    out, counts = restatement.integrate_direct(state, g["m"], 0.01, 1e-3, steps, integrator)
    for k in keys:
        assert np.array_equal(out[k], g[f"{tag}_{k}"]), k
    assert counts.evaluations == steps * (3 if integrator == "yoshida4" else 1)


def test_rk4_matches_reference_bitwise(restatement, golden_trajectory):
    # tests/golden/trajectory_rk4_512.npz: the reference's RungeKutta4
    # (runge_kutta4.cpp:64-139), 10 steps from the same start.
    g = golden_trajectory
    rk4 = dict(np.load(os.path.join(GOLDEN, "trajectory_rk4_512.npz")))
    keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
    state = {k: g[f"start_{k}"] for k in keys}
    out, counts = restatement.integrate_direct(state, g["m"], 0.01, 1e-3, 10, "rk4")
    for k in keys:
        assert np.array_equal(out[k], rk4[f"rk4_10_{k}"]), k
    assert counts.evaluations == 10 * 4


def test_rk4_matches_live_reference(restatement, reference):
    d = reference.plummer(257, 1.0, 1.0, 77)
    a0, _ = reference.direct(d["x"], d["y"], d["z"], d["m"], 0.02, kernel="scalar")
    state = dict(x=d["x"], y=d["y"], z=d["z"], vx=d["vx"], vy=d["vy"], vz=d["vz"],
                 ax=a0[:, 0].copy(), ay=a0[:, 1].copy(), az=a0[:, 2].copy())
    mine, _ = restatement.integrate_direct(state, d["m"], 0.02, 2e-3, 4, "rk4")
    theirs = reference.integrate_direct(state, d["m"], 0.02, 2e-3, 4, "rk4")
    assert all(np.array_equal(mine[k], theirs[k]) for k in state)


def test_energies_match_reference_bitwise(restatement, golden_plummer):
    g = golden_plummer
    assert restatement.potential_energy(g["x"], g["y"], g["z"], g["m"], 0.01) == \
        float(g["pe_eps0.01"])
    assert restatement.kinetic_energy(g["vx"], g["vy"], g["vz"], g["m"]) == float(g["ke"])


def test_yoshida_weights(restatement):
    outer, inner = restatement.yoshida_weights()
    assert abs(2 * outer + inner - 1.0) <= 4 * np.finfo(float).eps


# --------------------------------------------------------------------------
# Bit-for-bit against the live reference library (fresh seeds)
# --------------------------------------------------------------------------

@pytest.mark.parametrize("n,seed", [(1, 3), (33, 4), (700, 5), (5000, 6)])
def test_restatement_equals_reference_on_fresh_inputs(restatement, reference, n, seed):
    d = reference.plummer(n, 1.0, 1.0, seed)
    x, y, z, m = d["x"], d["y"], d["z"], d["m"]
    a_o, _ = restatement.direct(x, y, z, m, 0.02)
    a_r, _ = reference.direct(x, y, z, m, 0.02)
    assert np.array_equal(a_o, a_r)
    c_o, i_o, _, _ = restatement.morton_order(x, y, z)
    c_r, i_r, _, _ = reference.morton(x, y, z, threads=4)
    assert np.array_equal(c_o, c_r) and np.array_equal(i_o, i_r)
    for quad, leaf in ((False, 32), (True, 8)):
        a_o, c_o = restatement.barnes_hut(x, y, z, m, 0.02, 0.6, leaf, quad)
        a_r, c_r, _ = reference.barnes_hut(x, y, z, m, 0.02, 0.6, leaf, quad, with_tree=False)
        assert np.array_equal(a_o, a_r)
        assert [c_o.particle_particle, c_o.particle_cell] == c_r.tolist()[1:]


def test_reference_threads_do_not_change_the_tree(reference):
    # The reference's parallel tree build equals its serial build bit for bit
    # (tests/solvers/octree_test.cpp:453-492), so the serial restatement stands
    # for both.
    d = reference.plummer(60000, 1.0, 1.0, 20260810)
    a1, c1, t1 = reference.barnes_hut(d["x"], d["y"], d["z"], d["m"], 0.05, 0.5, 16, True,
                                      threads=1)
    a8, c8, t8 = reference.barnes_hut(d["x"], d["y"], d["z"], d["m"], 0.05, 0.5, 16, True,
                                      threads=8)
    assert np.array_equal(t1.reals, t8.reals) and np.array_equal(t1.idx, t8.idx)
    assert np.array_equal(t1.quads, t8.quads)
    assert np.array_equal(a1, a8) and np.array_equal(c1, c8)
