"""Checkpoint (ORRERYCK v1) and trajectory (ORRERYTJ v1) files from host arrays.

The reference's own writers and readers (src/sim/checkpoint.cpp,
src/sim/trajectory.cpp, compiled by the oracle recipe) are the parity bar:
this backend's files must equal theirs byte for byte for the same state, each
side must read the other's files, and damaged files must be refused. The
golden files under tests/golden/ were written by the reference
(tests/golden/make_golden_output.py) and pin the same bytes where the
reference library is not built. No GPU: the serializer is host code.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import orrery_b200 as ob

from conftest import GOLDEN

ARRAYS = ("m", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(ob.library_path()):
        from orrery_b200 import build
        build.build()
    return ob.load_library()


def state_of(n, seed=3, specials=True):
    rng = np.random.default_rng(seed)
    st = {k: rng.normal(size=n) for k in ARRAYS}
    st["m"] = rng.uniform(0.1, 2.0, n)
    if specials and n >= 4:
        # Bit patterns the format must carry exactly.
        st["x"][0] = -0.0
        st["vy"][1] = np.inf
        st["az"][2] = np.nan
        st["y"][3] = 5e-324  # the smallest subnormal
    return st


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def same_bits(a, b):
    return np.array_equal(bits(a), bits(b))


def read_bytes(path):
    with open(path, "rb") as f:
        return f.read()


# --------------------------------------------------------------------------
# Checkpoints
# --------------------------------------------------------------------------

@pytest.mark.parametrize("n", [0, 1, 257])
def test_checkpoint_bytes_equal_the_reference(lib, reference, tmp_path, n):
    st = state_of(n)
    text = reference.default_configuration()
    ours, theirs = tmp_path / "ours.ck", tmp_path / "theirs.ck"
    ob.write_checkpoint(ours, 1234, st, text)
    reference.write_checkpoint(theirs, 1234, st)
    assert read_bytes(ours) == read_bytes(theirs)
    assert not (tmp_path / "ours.ck.partial").exists()


def test_each_side_reads_the_others_checkpoint(lib, reference, tmp_path):
    st = state_of(300, seed=9)
    text = reference.default_configuration()
    ours, theirs = tmp_path / "ours.ck", tmp_path / "theirs.ck"
    ob.write_checkpoint(ours, 77, st, text)
    reference.write_checkpoint(theirs, 77, st)
    back = reference.read_checkpoint(ours)
    assert back["step"] == 77 and back["configuration"] == text
    assert all(same_bits(back[k], st[k]) for k in ARRAYS)
    mine = ob.read_checkpoint(theirs)
    assert mine["step"] == 77 and mine["configuration"] == text
    assert all(same_bits(mine[k], st[k]) for k in ARRAYS)
    assert ob.checkpoint_info(theirs) == {"step": 77, "n": 300,
                                          "configuration_bytes": len(text.encode())}


def test_golden_checkpoint_is_reproduced_and_read(lib, tmp_path):
    golden = os.path.join(GOLDEN, "checkpoint_64.orreryck")
    meta = dict(np.load(os.path.join(GOLDEN, "run_output_64.npz")))
    st = {k: meta[k] for k in ARRAYS}
    text = str(meta["configuration"])
    out = tmp_path / "again.ck"
    ob.write_checkpoint(out, int(meta["step"]), st, text)
    assert read_bytes(out) == read_bytes(golden)
    back = ob.read_checkpoint(golden)
    assert back["step"] == int(meta["step"]) and back["configuration"] == text
    assert all(same_bits(back[k], st[k]) for k in ARRAYS)


def _damaged(tmp_path, reference, edit):
    st = state_of(40)
    path = tmp_path / "d.ck"
    ob.write_checkpoint(path, 5, st, reference.default_configuration())
    data = bytearray(read_bytes(path))
    edit(data)
    bad = tmp_path / "bad.ck"
    bad.write_bytes(bytes(data))
    return bad


def _flip_state_byte(d):
    d[-100] ^= 0x01


def _set_version(d):
    d[8:12] = (2).to_bytes(4, "little")


def _set_flag(bit):
    def edit(d):
        d[12:16] = (1 << bit).to_bytes(4, "little")
    return edit


def _truncate(d):
    del d[-13:]


def _magic(d):
    d[0:8] = b"ORRERYTJ"


@pytest.mark.parametrize("edit", [_flip_state_byte, _set_version, _set_flag(0), _set_flag(5),
                                  _truncate, _magic],
                         ids=["bit-flip", "version", "single-precision", "unknown-flag",
                              "truncated", "magic"])
def test_damaged_checkpoints_are_refused_by_both_readers(lib, reference, tmp_path, edit):
    bad = _damaged(tmp_path, reference, edit)
    with pytest.raises(ob.OrreryError) as err:
        ob.read_checkpoint(bad)
    assert err.value.code == ob.ERROR_IO
    with pytest.raises(RuntimeError):
        reference.read_checkpoint(bad)


def test_unwritable_checkpoint_path_is_an_io_error(lib, tmp_path):
    with pytest.raises(ob.OrreryError) as err:
        ob.write_checkpoint(tmp_path / "missing" / "x.ck", 1, state_of(4), "")
    assert err.value.code == ob.ERROR_IO


def test_rewriting_replaces_the_previous_checkpoint(lib, tmp_path):
    path = tmp_path / "run.ck"
    ob.write_checkpoint(path, 1, state_of(16, seed=1), "a")
    ob.write_checkpoint(path, 2, state_of(16, seed=2), "b")
    back = ob.read_checkpoint(path)
    assert back["step"] == 2 and back["configuration"] == "b"
    assert same_bits(back["x"], state_of(16, seed=2)["x"])
    assert sorted(p.name for p in tmp_path.iterdir()) == ["run.ck"]


# --------------------------------------------------------------------------
# Trajectories
# --------------------------------------------------------------------------

def frames_of(n, count, seed=4):
    out = []
    for f in range(count):
        st = state_of(n, seed=seed + f, specials=f == 0)
        out.append((10 * f, 10 * f * 1e-3, st))
    return out


@pytest.mark.parametrize("n,with_velocities", [(0, False), (1, True), (129, False), (129, True)])
def test_trajectory_bytes_equal_the_reference(lib, reference, tmp_path, n, with_velocities):
    masses = state_of(n)["m"]
    frames = frames_of(n, 3)
    ours, theirs = tmp_path / "ours.tj", tmp_path / "theirs.tj"
    with ob.Trajectory(ours, 1e-3, masses=masses, with_velocities=with_velocities) as t:
        for step, time, st in frames:
            t.write_frame(step, time, st)
        assert t.frames == 3
    reference.write_trajectory(theirs, masses, 1e-3, frames, with_velocities)
    assert read_bytes(ours) == read_bytes(theirs)


def test_reference_reads_our_trajectory(lib, reference, tmp_path):
    masses = state_of(50)["m"]
    frames = frames_of(50, 4)
    path = tmp_path / "t.tj"
    with ob.Trajectory(path, 2.5e-4, masses=masses, with_velocities=True) as t:
        for step, time, st in frames:
            t.write_frame(step, time, st)
    got = reference.read_trajectory(path)
    assert got["n"] == 50 and got["timestep"] == 2.5e-4 and got["with_velocities"]
    assert same_bits(got["masses"], masses) and got["frame_count"] == 4
    for (step, time, st), (s2, t2, st2) in zip(frames, got["frames"]):
        assert step == s2 and time == t2
        assert all(same_bits(st[k], st2[k]) for k in ("x", "y", "z", "vx", "vy", "vz"))


def test_golden_trajectory_is_reproduced(lib, tmp_path):
    meta = dict(np.load(os.path.join(GOLDEN, "run_output_64.npz")))
    n = len(meta["m"])
    out = tmp_path / "again.tj"
    with ob.Trajectory(out, float(meta["timestep"]), masses=meta["m"], with_velocities=True) as t:
        for f in range(int(meta["frames"])):
            st = {k: meta[f"frame{f}_{k}"] for k in ("x", "y", "z", "vx", "vy", "vz")}
            t.write_frame(int(meta["frame_steps"][f]), float(meta["frame_times"][f]), st)
    assert read_bytes(out) == read_bytes(os.path.join(GOLDEN, "trajectory_64.orrerytj"))
    assert n == 64


def test_trajectory_frame_needs_its_arrays(lib, tmp_path):
    with ob.Trajectory(tmp_path / "t.tj", 1e-3, masses=np.ones(8), with_velocities=True) as t:
        with pytest.raises(KeyError):
            t.write_frame(0, 0.0, {"x": np.zeros(8), "y": np.zeros(8), "z": np.zeros(8)})
    with pytest.raises(ob.OrreryError) as err:
        ob.Trajectory(tmp_path / "nowhere" / "t.tj", 1e-3, masses=np.ones(2))
    assert err.value.code == ob.ERROR_IO
