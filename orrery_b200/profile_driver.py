"""Small, fixed workloads for profiling one kernel at a time.

    python -m orrery_b200.profile_driver tree N      # Barnes-Hut evaluations of the
                                                     # two-disc collision of N particles
    python -m orrery_b200.profile_driver pack        # FP32 direct solver, Plummer 262,144
    python -m orrery_b200.profile_driver batch       # 64 clusters (3 above 8192 particles)
                                                     # in chunked batched items
    python -m orrery_b200.profile_driver rk4         # two RK4 steps, Plummer 1,048,576
    python -m orrery_b200.profile_driver fused       # FP32 direct system of 4096 particles:
                                                     # single-launch velocity-Verlet steps

Each runs a handful of launches of the kernels it names, on seeded synthetic
inputs, and exits 0; a profiler then captures the launches it wants (for
example `ncu -k regex:walk_kernel -s 2 -c 1`).
"""
from __future__ import annotations

import sys

import numpy as np

from . import initial_conditions as ic


def tree(n: int) -> None:
    from . import B200TreeSolver

    d = ic.galaxy_collision(n, softening=0.02, seed=20260811)
    solver = B200TreeSolver(0.02, 0.5, 32, True)
    for _ in range(4):
        solver.evaluate((d["x"], d["y"], d["z"]), d["m"])


def pack() -> None:
    from . import B200DirectSolver

    d = ic.plummer_sphere(262144, seed=5)
    solver = B200DirectSolver(0.01, "fp32")
    for _ in range(3):
        solver.evaluate((d["x"], d["y"], d["z"]), d["m"])


def batch() -> None:
    from . import DeviceBatch

    rng = np.random.default_rng(41)
    sizes = np.concatenate([[16384, 12288, 9001],
                            np.exp(rng.uniform(np.log(256), np.log(16384), 61)).astype(int)])
    radii = rng.uniform(0.5, 2.0, len(sizes))
    b = DeviceBatch(sizes, 0.01 * radii)
    b.set_shape(256, 4, 4, 8)  # chunks of 4 source tiles: partial sums and their reduction
    for k, n in enumerate(sizes):
        d = ic.plummer_sphere(int(n), scale_radius=float(radii[k]), seed=100 + k)
        b.set_state(k, d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    b.refresh()
    b.step(1e-3, 2, "yoshida4")


def rk4() -> None:
    from . import DeviceSystem

    n = 1 << 20
    d = ic.plummer_sphere(n, seed=6)
    system = DeviceSystem(n, 0.01, precision="fp32")
    system.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    system.step(1e-4, 2, "rk4")


def fused() -> None:
    from . import DeviceSystem

    n = 4096
    d = ic.plummer_sphere(n, seed=7)
    system = DeviceSystem(n, 0.01, precision="fp32")
    if not system.set_fused_steps(True):
        raise SystemExit("the single-launch steps do not apply to this system")
    system.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    for _ in range(4):
        system.step(1e-3, 1, "vv")


def main(argv: list[str]) -> None:
    from . import load_library

    load_library()
    what = argv[1] if len(argv) > 1 else ""
    if what == "tree":
        tree(int(argv[2]))
    elif what in ("pack", "batch", "rk4", "fused"):
        {"pack": pack, "batch": batch, "rk4": rk4, "fused": fused}[what]()
    else:
        raise SystemExit(__doc__)
    print("ok", what)


if __name__ == "__main__":
    main(sys.argv)
