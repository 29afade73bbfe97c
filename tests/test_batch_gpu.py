"""Batched form: many systems of uneven size, each with its own softening, in
one persistent launch.

Each system's forces are held to the precision form's bounds against the FP64
oracle run on that system alone with its own softening; a system's result is
bit-identical whether it is alone or in the batch (its work items and their
arithmetic do not depend on the other systems); Yoshida-4 steps of the batch
agree with the same systems stepped one at a time by the single-system
precision path.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import relative_errors

pytestmark = pytest.mark.gpu

SPLIT_WORST, SPLIT_MEDIAN = 2e-6, 1e-7


def _systems(count, seed, lo=256, hi=4000):
    from orrery_b200 import initial_conditions as ic
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
    radii = rng.uniform(0.5, 2.0, count)
    systems = [ic.plummer_sphere(int(n), scale_radius=float(a), seed=seed * 1000 + k)
               for k, (n, a) in enumerate(zip(sizes, radii))]
    return sizes, radii, systems


def _batch(b200, sizes, radii, systems):
    batch = b200.DeviceBatch(sizes, 0.01 * radii)
    for k, d in enumerate(systems):
        batch.set_state(k, d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    batch.refresh()
    return batch


def test_every_system_matches_the_fp64_oracle(b200, restatement):
    sizes, radii, systems = _systems(20, 3)
    batch = _batch(b200, sizes, radii, systems)
    for k, d in enumerate(systems):
        st = batch.state(k)
        a = np.stack([st["ax"], st["ay"], st["az"]], axis=1)
        exact, _ = restatement.direct(d["x"], d["y"], d["z"], d["m"], 0.01 * radii[k])
        err = relative_errors(a, exact)
        assert err.max() < SPLIT_WORST, (k, err.max())
        assert np.median(err) < SPLIT_MEDIAN
    pairs, evals, items = batch.stats()
    assert pairs == sum(int(n) * (int(n) - 1) for n in sizes) and evals == 1


@pytest.fixture(scope="module")
def full_range(restatement):
    """The batched configuration's whole size range, [256, 16384]: its two
    ends, three systems above 8192 (whose sources span 17 to 32 tiles of 512)
    and log-uniform draws between, each with its own scale radius and
    softening 0.01 x radius; with the FP64 oracle's accelerations."""
    from orrery_b200 import initial_conditions as ic
    rng = np.random.default_rng(41)
    sizes = np.concatenate([[256, 16384, 12288, 9001],
                            np.exp(rng.uniform(np.log(256), np.log(16384), 8)).astype(int)])
    radii = rng.uniform(0.5, 2.0, len(sizes))
    systems = [ic.plummer_sphere(int(n), scale_radius=float(a), seed=4100 + k)
               for k, (n, a) in enumerate(zip(sizes, radii))]
    exact = [restatement.direct(d["x"], d["y"], d["z"], d["m"], 0.01 * radii[k])[0]
             for k, d in enumerate(systems)]
    return sizes, radii, systems, exact


# Default items (a whole system's sources each) and chunked items of 4 and 8
# source tiles, whose partial sums batch_reduce_kernel adds in chunk order.
@pytest.mark.parametrize("shape", [None, (256, 4, 4, 8), (128, 2, 8, 4)])
def test_the_full_size_range_matches_the_fp64_oracle(b200, full_range, shape):
    sizes, radii, systems, exact = full_range
    assert sizes.min() == 256 and sizes.max() == 16384 and (sizes > 8192).sum() >= 3
    batch = b200.DeviceBatch(sizes, 0.01 * radii)
    if shape is not None:
        batch.set_shape(*shape)
    for k, d in enumerate(systems):
        batch.set_state(k, d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    batch.refresh()
    for k in range(len(systems)):
        st = batch.state(k)
        a = np.stack([st["ax"], st["ay"], st["az"]], axis=1)
        err = relative_errors(a, exact[k])
        assert np.median(err) < SPLIT_MEDIAN, (k, int(sizes[k]))
        # Per particle the FP32 term roundings (~1e-7 each) add up relative to
        # the terms' magnitudes, not to their sum: where the net force nearly
        # cancels (near a cluster's centre, |a| -> 0) the relative error grows
        # with the cancellation. Measured against max(|a_i|, median |a|) the
        # bound is the precision form's; the plain relative error stays
        # within 1e-5 for every particle.
        mag = np.linalg.norm(exact[k], axis=1)
        scale = np.maximum(mag, np.median(mag))
        normwise = np.linalg.norm(a - exact[k], axis=1) / scale
        assert normwise.max() < SPLIT_WORST, (k, int(sizes[k]), normwise.max(), err.max())
        assert err.max() < 1e-5, (k, int(sizes[k]), err.max())


@pytest.mark.parametrize("shape", [(128, 2, 0), (128, 2, 4), (128, 4, 1), (256, 2, 0),
                                   (256, 4, 2), (128, 2, 0, 4), (256, 2, 4, 8), (256, 4, 0, 4),
                                   (256, 4, 2, 8)])
def test_every_shape_computes_the_same_sums(b200, restatement, shape):
    sizes, radii, systems = _systems(9, 5, hi=6000)
    batch = b200.DeviceBatch(sizes, 0.01 * radii)
    batch.set_shape(*shape)
    for k, d in enumerate(systems):
        batch.set_state(k, d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    batch.refresh()
    for k in (0, 4, 8):
        d = systems[k]
        st = batch.state(k)
        exact, _ = restatement.direct(d["x"], d["y"], d["z"], d["m"], 0.01 * radii[k])
        a = np.stack([st["ax"], st["ay"], st["az"]], axis=1)
        assert relative_errors(a, exact).max() < SPLIT_WORST


def test_a_system_is_bit_identical_alone_and_in_the_mix(b200):
    sizes, radii, systems = _systems(12, 7)
    mix = _batch(b200, sizes, radii, systems)
    for k in (0, 5, 11):
        alone = _batch(b200, sizes[k:k + 1], radii[k:k + 1], systems[k:k + 1])
        a, b = mix.state(k), alone.state(0)
        assert all(np.array_equal(a[c], b[c]) for c in ("ax", "ay", "az"))
    mix.step(1e-3, 3, "yoshida4")
    alone = _batch(b200, sizes[5:6], radii[5:6], systems[5:6])
    alone.step(1e-3, 3, "yoshida4")
    a, b = mix.state(5), alone.state(0)
    assert all(np.array_equal(a[c], b[c]) for c in b200.DeviceBatch.KEYS)


def test_batched_yoshida_steps_track_single_system_steps(b200):
    sizes, radii, systems = _systems(6, 9, hi=3000)
    batch = _batch(b200, sizes, radii, systems)
    batch.step(1e-3, 10, "yoshida4")
    for k, d in enumerate(systems):
        single = b200.DeviceSystem(int(sizes[k]), 0.01 * radii[k], precision="split")
        single.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
        single.step(1e-3, 10, "yoshida4")
        a, b = batch.state(k), single.state()
        assert np.max(np.abs(a["x"] - b["x"])) < 1e-9
        assert np.max(np.abs(a["vz"] - b["vz"])) < 1e-8


def test_energy_is_conserved_per_system(b200):
    sizes, radii, systems = _systems(4, 11, hi=2000)
    batch = _batch(b200, sizes, radii, systems)
    e0 = [sum(batch.energy(k)) for k in range(4)]
    batch.step(1e-3, 50, "yoshida4")
    for k in range(4):
        e = sum(batch.energy(k))
        assert abs(e - e0[k]) / abs(e0[k]) < 1e-6


def test_batches_refuse_rk4(b200):
    batch = b200.DeviceBatch([600], [0.01])
    with pytest.raises(b200.OrreryError) as err:
        batch.step(1e-3, 1, "rk4")
    assert err.value.code == b200.ERROR_UNSUPPORTED


def test_mass_beyond_the_fp32_range_is_refused(b200):
    # The batched kernel adds a target's own entry as f * 0 with f = m / eps^3
    # in FP32: a mass that makes f overflow would turn that zero into NaN.
    batch = b200.DeviceBatch([600], [0.01])
    x, y, z = (np.linspace(0.0, 1.0, 600) + k for k in range(3))
    with pytest.raises(b200.OrreryError):
        batch.set_state(0, x, y, z, None, None, None, np.full(600, 1e32))
    batch.set_state(0, x, y, z, None, None, None, np.full(600, 1e30))


def test_autotune_keeps_results_within_bounds(b200, restatement):
    sizes, radii, systems = _systems(16, 13, hi=8000)
    batch = _batch(b200, sizes, radii, systems)
    shape, ms = batch.autotune()
    assert ms > 0
    d = systems[3]
    st = batch.state(3)
    exact, _ = restatement.direct(d["x"], d["y"], d["z"], d["m"], 0.01 * radii[3])
    a = np.stack([st["ax"], st["ay"], st["az"]], axis=1)
    assert relative_errors(a, exact).max() < SPLIT_WORST


def test_invalid_batches_are_refused(b200):
    with pytest.raises(b200.OrreryError):
        b200.DeviceBatch([100, 200], [0.01, 0.0])   # a zero softening
    with pytest.raises(b200.OrreryError):
        b200.DeviceBatch([100, 0], [0.01, 0.01])    # an empty system
