"""Generates the run-output golden files in this directory with the reference.

Run in a checkout where the reference's sources exist (the oracle Makefile
compiles them, src/sim/checkpoint.cpp and src/sim/trajectory.cpp included,
into oracle/_ref/libref_orrery.so):

    python tests/golden/make_golden_output.py

Writes, for 64 particles of seeded state (a few special bit patterns
included: -0, +inf, a NaN, the smallest subnormal):

* checkpoint_64.orreryck -- sim::write_checkpoint of {the reference's default
  Configuration, step 4321, the state};
* trajectory_64.orrerytj -- sim::TrajectoryWriter with velocities, timestep
  5e-4, three frames;
* run_output_64.npz      -- the inputs of both: the ten state arrays, the step,
  the configuration text the reference wrote, the timestep and the frames.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

ARRAYS = ("m", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
N, STEP, TIMESTEP, FRAMES = 64, 4321, 5e-4, 3


def main() -> None:
    oracle.build()
    ref = oracle.Reference()
    rng = np.random.default_rng(20260903)
    st = {k: rng.normal(size=N) for k in ARRAYS}
    st["m"] = rng.uniform(0.1, 2.0, N)
    st["x"][0] = -0.0
    st["vy"][1] = np.inf
    st["az"][2] = np.nan
    st["y"][3] = 5e-324
    ref.write_checkpoint(os.path.join(HERE, "checkpoint_64.orreryck"), STEP, st)
    frames = []
    for f in range(FRAMES):
        fr = {k: rng.normal(size=N) for k in ("x", "y", "z", "vx", "vy", "vz")}
        frames.append((100 * f, 100 * f * TIMESTEP, fr))
    ref.write_trajectory(os.path.join(HERE, "trajectory_64.orrerytj"), st["m"], TIMESTEP, frames,
                         True)
    extra = {f"frame{f}_{k}": frames[f][2][k] for f in range(FRAMES) for k in frames[f][2]}
    np.savez(os.path.join(HERE, "run_output_64.npz"), **st, step=STEP,
             configuration=np.array(ref.default_configuration()), timestep=TIMESTEP,
             frames=FRAMES, frame_steps=np.array([f[0] for f in frames], dtype=np.uint64),
             frame_times=np.array([f[1] for f in frames]), **extra)


if __name__ == "__main__":
    main()
