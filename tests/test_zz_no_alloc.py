"""The allocation-free ordering entry point, ob_morton_order_noalloc.

It exists for callers that cannot allocate device memory at the moment they
need an ordering (services limited to their own fixed pool of device memory,
or that must not grow the device heap once running): it takes device inputs
and outputs and keeps every intermediate buffer in a fixed device array.
These checks call it through the C ABI twice in a row, on different inputs,
and hold each result to the ordering the tree solver's own pipeline produces
for the same particles and to the oracle's MortonOrdering restatement --
integer outputs, so the tolerance is equality -- with its status word
reporting success; and check that a request above its fixed capacity is
refused. This file is collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CAPACITY = 1 << 20


def _entry(b200):
    lib = b200.load_library()
    fn = lib.ob_morton_order_noalloc
    fn.argtypes = [C.c_uint64] + [C.c_void_p] * 7
    fn.restype = C.c_int
    return lib, fn


def test_noalloc_ordering_equals_the_tree_solvers_ordering(b200, restatement):
    torch = pytest.importorskip("torch")
    from orrery_b200 import initial_conditions as ic

    lib, fn = _entry(b200)
    device = torch.device("cuda:0")
    for seed, n in ((11, 300_000), (12, 77_777)):
        d = ic.plummer_sphere(n, seed=seed)
        xs = [torch.tensor(d[k], dtype=torch.float64, device=device) for k in ("x", "y", "z")]
        codes = torch.empty(n, dtype=torch.int64, device=device)
        indices = torch.empty(n, dtype=torch.int32, device=device)
        status = torch.full((1,), 0x5a5a5a5a, dtype=torch.int32, device=device)
        stream = torch.cuda.current_stream(device).cuda_stream
        rc = fn(n, *(t.data_ptr() for t in xs), codes.data_ptr(), indices.data_ptr(),
                status.data_ptr(), stream)
        assert rc == b200.OK, lib.ob_last_error()
        torch.cuda.synchronize(device)
        assert int(status.item()) == 0
        got_codes = codes.cpu().numpy().view(np.uint64)
        got_indices = indices.cpu().numpy().view(np.uint32)

        solver = b200.B200TreeSolver(0.02, 0.5, 32, False)
        solver.evaluate((d["x"], d["y"], d["z"]), d["m"])
        want_codes, want_indices, _, _ = solver.order(n)
        assert np.array_equal(got_codes, want_codes)
        assert np.array_equal(got_indices, want_indices)
        if n <= 100_000:
            oracle_codes, oracle_indices = restatement.morton_order(d["x"], d["y"], d["z"])[:2]
            assert np.array_equal(got_codes, oracle_codes)
            assert np.array_equal(got_indices, oracle_indices)


def test_noalloc_ordering_refuses_more_than_its_capacity(b200):
    lib, fn = _entry(b200)
    rc = fn(CAPACITY + 1, None, None, None, None, None, None, None)
    assert rc == b200.ERROR_CAPACITY
    assert b"1048576" in lib.ob_last_error()
