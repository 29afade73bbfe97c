"""Generates trajectory_rk4_512.npz with the reference's own RungeKutta4.

Run where the reference's sources exist (the oracle Makefile compiles
src/integrators/runge_kutta4.cpp into oracle/_ref/libref_orrery.so):

    python tests/golden/make_golden_rk4.py

Starts from the 512-particle state of trajectory_512.npz (a Plummer sphere from
the reference's generator, its FP64 scalar direct accelerations) and takes 10
RK4 steps of dt 1e-3 with the FP64 scalar DirectSolver, eps 0.01.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def main() -> None:
    oracle.build()
    ref = oracle.Reference()
    g = dict(np.load(os.path.join(HERE, "trajectory_512.npz")))
    state = {k: g[f"start_{k}"] for k in KEYS}
    out = ref.integrate_direct(state, g["m"], 0.01, 1e-3, 10, "rk4")
    np.savez_compressed(os.path.join(HERE, "trajectory_rk4_512.npz"),
                        **{f"rk4_10_{k}": out[k] for k in KEYS})


if __name__ == "__main__":
    main()
