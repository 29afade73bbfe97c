"""Generates the golden fixtures in this directory from the reference itself.

Run in a checkout where the reference's sources exist (the oracle Makefile
compiles them into oracle/_ref/libref_orrery.so):

    python tests/golden/make_golden.py

Every array in the fixtures is an output of the reference's own C++ classes
(make_plummer_sphere, DirectSolver, BarnesHutSolver, MortonOrdering,
VelocityVerlet, Yoshida4, potential_energy) on seeded inputs. The fixtures let
the GPU tests compare against the reference where its sources are absent.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

SEED = 20260811  # the reference's CUDA-test seed (tests/solvers/cuda_direct_solver_test.cpp:71)


def main() -> None:
    oracle.build()
    ref = oracle.Reference()

    # Forces, Morton order and trees on a 2048-particle Plummer sphere.
    n = 2048
    d = ref.plummer(n, 1.0, 1.0, SEED)
    x, y, z, m = d["x"], d["y"], d["z"], d["m"]
    out = dict(x=x, y=y, z=z, vx=d["vx"], vy=d["vy"], vz=d["vz"], m=m)
    for eps in (0.01, 0.05):
        a, pairs = ref.direct(x, y, z, m, eps, kernel="scalar")
        out[f"direct_eps{eps}"] = a
        out["direct_pairs"] = np.uint64(pairs)
    codes, idx, origin, size = ref.morton(x, y, z)
    out.update(morton_codes=codes, morton_index=idx, cube_origin=origin, cube_size=size)
    for quad in (False, True):
        tag = "quad" if quad else "mono"
        a, counts, tree = ref.barnes_hut(x, y, z, m, 0.05, 0.5, 32, quad)
        out[f"bh_{tag}_acc"] = a
        out[f"bh_{tag}_counts"] = counts
        out[f"bh_{tag}_reals"] = tree.reals
        out[f"bh_{tag}_idx"] = tree.idx
        out[f"bh_{tag}_meta"] = np.array([tree.leaf_count, tree.depth], np.uint64)
        if quad:
            out["bh_quad_quads"] = tree.quads
    a, counts, tree = ref.barnes_hut(x, y, z, m, 0.05, 0.0, 32, False)
    out["bh_theta0_acc"] = a
    out["bh_theta0_counts"] = counts
    out["pe_eps0.01"] = ref.potential_energy(x, y, z, m, 0.01)
    out["ke"] = ref.kinetic_energy(d["vx"], d["vy"], d["vz"], m)
    np.savez_compressed(os.path.join(HERE, "plummer_2048.npz"), **out)

    # Integrator trajectories on a 512-particle sphere: FP64 scalar direct
    # field, velocity Verlet and Yoshida-4, dt 1e-3, eps 0.01.
    n = 512
    d = ref.plummer(n, 1.0, 1.0, SEED + 1)
    a0, _ = ref.direct(d["x"], d["y"], d["z"], d["m"], 0.01, kernel="scalar")
    state = dict(x=d["x"], y=d["y"], z=d["z"], vx=d["vx"], vy=d["vy"], vz=d["vz"],
                 ax=a0[:, 0].copy(), ay=a0[:, 1].copy(), az=a0[:, 2].copy())
    traj = {f"start_{k}": v for k, v in state.items()}
    traj["m"] = d["m"]
    vv = ref.integrate_direct(state, d["m"], 0.01, 1e-3, 20, "vv")
    y4 = ref.integrate_direct(state, d["m"], 0.01, 1e-3, 10, "yoshida4")
    for k in state:
        traj[f"vv20_{k}"] = vv[k]
        traj[f"y4_10_{k}"] = y4[k]
    np.savez_compressed(os.path.join(HERE, "trajectory_512.npz"), **traj)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
