"""orrery_b200: a B200 (sm_100a) force-evaluation backend for Orrery.

Python view of the C ABI in ``include/orrery_b200.h``. The solver classes
mirror the reference's ``ForceSolver`` surface
(include/orrery/solvers/force_solver.hpp:41-87): ``evaluate(positions, masses,
accelerations)`` writes accelerations for FP64 structure-of-arrays input,
``name()``, ``softening()``, ``interaction_count()`` and
``reset_interaction_count()``; construction goes through ``try_create``, which
returns ``None`` when no usable device exists, as ``CudaDirectSolver::try_create``
does (src/solvers/cuda_direct_solver.cpp:140-164). Runtime failures raise
:class:`OrreryError` carrying the C status code.

There is no CPU fallback: importing works without a GPU (so that host logic can
be tested), but every call that needs the device goes through the CUDA library
and fails with an error when the library or the device is missing.
"""
from __future__ import annotations

import ctypes as C
import operator
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(HERE, "_lib", "liborrery_b200.so")

OK = 0
ERROR_INVALID_ARGUMENT = 1
ERROR_NO_DEVICE = 2
ERROR_OUT_OF_MEMORY = 3
ERROR_CUDA = 4
ERROR_TIMEOUT = 5
ERROR_CAPACITY = 6
ERROR_UNSUPPORTED = 7
ERROR_IO = 8

SOLVER_DIRECT = 0
SOLVER_TREE = 1
PRECISION_FP32 = 0
PRECISION_SPLIT = 1
PRECISION_FP64 = 2
INTEGRATOR_VV = 0
INTEGRATOR_YOSHIDA4 = 1
INTEGRATOR_RK4 = 2

_PRECISIONS = {"fp32": PRECISION_FP32, "split": PRECISION_SPLIT, "fp64": PRECISION_FP64}
_INTEGRATORS = {"vv": INTEGRATOR_VV, "velocity-verlet": INTEGRATOR_VV,
                "yoshida4": INTEGRATOR_YOSHIDA4, "rk4": INTEGRATOR_RK4,
                "runge-kutta4": INTEGRATOR_RK4}


class OrreryError(RuntimeError):
    """A failed C-ABI call: ``code`` is the OB_ERROR_* status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class SolverParams(C.Structure):
    _fields_ = [("kind", C.c_int32), ("precision", C.c_int32), ("softening_squared", C.c_double),
                ("opening_angle", C.c_double), ("leaf_capacity", C.c_uint64),
                ("quadrupole", C.c_int32), ("reserved", C.c_int32)]


class Counts(C.Structure):
    _fields_ = [("evaluations", C.c_uint64), ("particle_particle", C.c_uint64),
                ("particle_cell", C.c_uint64)]


class DirectShape(C.Structure):
    _fields_ = [("threads", C.c_int32), ("targets_per_thread", C.c_int32),
                ("split", C.c_int32), ("groups", C.c_int32)]


class BatchShape(C.Structure):
    _fields_ = [("threads", C.c_int32), ("targets_per_thread", C.c_int32),
                ("chunk_tiles", C.c_uint32), ("groups", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("direct_pairs_cap", C.c_uint64),
                ("direct_arena_particles", C.c_uint64), ("max_tree_jobs", C.c_uint32),
                ("fake_device", C.c_int32), ("fake_direct_gint_s", C.c_double),
                ("fake_tree_ns_per_particle", C.c_double), ("max_job_work", C.c_double),
                ("max_running_work", C.c_double)]


class JobSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("integrator", C.c_int32), ("n", C.c_uint64),
                ("steps", C.c_uint64), ("dt", C.c_double), ("softening_squared", C.c_double),
                ("opening_angle", C.c_double), ("leaf_capacity", C.c_uint64),
                ("quadrupole", C.c_int32), ("reserved", C.c_int32)]


class JobReport(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int32), ("reserved", C.c_int32),
                ("steps_done", C.c_uint64), ("submitted_s", C.c_double),
                ("admitted_s", C.c_double), ("finished_s", C.c_double)]


class ServerSummary(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("failed", C.c_uint64), ("cancelled", C.c_uint64), ("rejected", C.c_uint64),
                ("queued", C.c_uint64), ("running", C.c_uint64), ("elapsed_s", C.c_double),
                ("jobs_per_s", C.c_double), ("job_latency_p50_s", C.c_double),
                ("job_latency_p99_s", C.c_double), ("step_latency_p50_ms", C.c_double),
                ("step_latency_p99_ms", C.c_double), ("hbm_in_use", C.c_uint64),
                ("hbm_peak", C.c_uint64)]


class DiagnosticsRecord(C.Structure):
    """ob_diagnostics, as the C ABI fills it."""

    _fields_ = [("kinetic_energy", C.c_double), ("potential_energy", C.c_double),
                ("linear_momentum", C.c_double * 3), ("angular_momentum", C.c_double * 3)]


class Timings(C.Structure):
    _fields_ = [("transfer_in_ms", C.c_double), ("ordering_ms", C.c_double),
                ("construction_ms", C.c_double), ("traversal_ms", C.c_double),
                ("transfer_out_ms", C.c_double)]


@dataclass
class InteractionCount:
    """solvers::InteractionCount (include/orrery/solvers/interaction_count.hpp:37-76)."""
    evaluations: int = 0
    particle_particle: int = 0
    particle_cell: int = 0


_dp = C.POINTER(C.c_double)
_lib = None


def library_path() -> str:
    return LIBRARY_PATH


def load_library():
    """Loads the CUDA library, raising if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY_PATH):
        raise OrreryError(ERROR_NO_DEVICE,
                          f"the CUDA library is missing ({LIBRARY_PATH}); run "
                          "`python -m orrery_b200.build`")
    lib = C.CDLL(LIBRARY_PATH)
    vp = C.c_void_p
    lib.ob_version.restype = C.c_char_p
    lib.ob_last_error.restype = C.c_char_p
    lib.ob_device_count.argtypes = [C.POINTER(C.c_int)]
    lib.ob_solver_create.argtypes = [C.POINTER(SolverParams), C.POINTER(vp)]
    lib.ob_solver_destroy.argtypes = [vp]
    lib.ob_solver_destroy.restype = None
    lib.ob_solver_get_params.argtypes = [vp, C.POINTER(SolverParams)]
    lib.ob_solver_evaluate.argtypes = [vp, C.c_uint64] + [_dp] * 7
    lib.ob_solver_evaluate_device.argtypes = [vp, C.c_uint64] + [vp] * 7 + [vp]
    lib.ob_solver_counts.argtypes = [vp, C.POINTER(Counts)]
    lib.ob_solver_reset_counts.argtypes = [vp]
    lib.ob_solver_timings.argtypes = [vp, C.POINTER(Timings)]
    lib.ob_direct_shapes.argtypes = [C.c_int32, C.POINTER(DirectShape), C.c_int32,
                                     C.POINTER(C.c_int32)]
    lib.ob_solver_set_direct_shape.argtypes = [vp, C.c_uint64, C.POINTER(DirectShape)]
    lib.ob_solver_autotune.argtypes = [vp, C.c_uint64, C.POINTER(DirectShape),
                                       C.POINTER(C.c_double)]
    lib.ob_system_create.argtypes = [C.POINTER(SolverParams), C.c_uint64, C.POINTER(vp)]
    lib.ob_system_destroy.argtypes = [vp]
    lib.ob_system_destroy.restype = None
    lib.ob_system_set_state.argtypes = [vp] + [_dp] * 7
    lib.ob_system_set_accelerations.argtypes = [vp] + [_dp] * 3
    lib.ob_system_get_state.argtypes = [vp] + [_dp] * 9
    lib.ob_system_step_host.argtypes = [vp, C.c_int32, C.c_double, C.c_uint64] + [_dp] * 10
    lib.ob_system_step.argtypes = [vp, C.c_int32, C.c_double, C.c_uint64]
    lib.ob_system_step_async.argtypes = [vp, C.c_int32, C.c_double, C.c_uint64]
    lib.ob_system_synchronize.argtypes = [vp]
    lib.ob_system_energy.argtypes = [vp, _dp, _dp]
    lib.ob_system_counts.argtypes = [vp, C.POINTER(Counts)]
    lib.ob_system_size.argtypes = [vp, C.POINTER(C.c_uint64)]
    lib.ob_probe_fp32.argtypes = [_dp, _dp]
    lib.ob_probe_fp32x2.argtypes = [_dp]
    lib.ob_probe_fp64.argtypes = [_dp]
    lib.ob_system_diagnostics.argtypes = [vp, C.POINTER(DiagnosticsRecord)]
    lib.ob_system_device_arrays.argtypes = [vp, C.POINTER(vp)]
    lib.ob_system_snapshot.argtypes = [vp] + [_dp] * 10
    lib.ob_system_restore.argtypes = [vp] + [_dp] * 10
    _u64p = C.POINTER(C.c_uint64)
    lib.ob_tree_stats.argtypes = [vp, _u64p, _u64p, C.POINTER(C.c_uint32)]
    lib.ob_tree_copy.argtypes = [vp, _dp, _u64p, _dp]
    lib.ob_tree_copy_order.argtypes = [vp, _u64p, C.POINTER(C.c_uint32), _dp, _dp]
    lib.ob_system_stream.argtypes = [vp, C.POINTER(vp)]
    lib.ob_system_autotune.argtypes = [vp, C.POINTER(DirectShape), C.POINTER(C.c_double)]
    lib.ob_system_profile.argtypes = [vp, C.c_uint32]
    lib.ob_system_phase_times.argtypes = [vp, C.POINTER(Timings), C.POINTER(C.c_uint32)]
    lib.ob_system_step_kernels.argtypes = [vp, C.c_int32, C.c_double, C.POINTER(C.c_uint32)]
    lib.ob_system_set_fused_steps.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32)]
    lib.ob_batch_create.argtypes = [C.c_uint32, C.POINTER(C.c_uint64), _dp, C.POINTER(vp)]
    lib.ob_batch_destroy.argtypes = [vp]
    lib.ob_batch_destroy.restype = None
    lib.ob_batch_set_state.argtypes = [vp, C.c_uint32] + [_dp] * 7
    lib.ob_batch_get_state.argtypes = [vp, C.c_uint32] + [_dp] * 9
    lib.ob_batch_refresh.argtypes = [vp]
    lib.ob_batch_step.argtypes = [vp, C.c_int32, C.c_double, C.c_uint64]
    lib.ob_batch_step_async.argtypes = [vp, C.c_int32, C.c_double, C.c_uint64]
    lib.ob_batch_synchronize.argtypes = [vp]
    lib.ob_batch_energy.argtypes = [vp, C.c_uint32, _dp, _dp]
    lib.ob_batch_autotune.argtypes = [vp, C.POINTER(BatchShape), C.POINTER(C.c_double)]
    lib.ob_batch_set_shape.argtypes = [vp, C.POINTER(BatchShape)]
    lib.ob_batch_stats.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint32)]
    lib.ob_batch_stream.argtypes = [vp, C.POINTER(vp)]
    lib.ob_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(vp)]
    lib.ob_server_destroy.argtypes = [vp]
    lib.ob_server_destroy.restype = None
    lib.ob_server_submit.argtypes = [vp, C.POINTER(JobSpec)] + [_dp] * 7 + [
        C.POINTER(C.c_uint64)]
    lib.ob_server_wait.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(JobReport)] + [_dp] * 9
    lib.ob_server_cancel.argtypes = [vp, C.c_uint64]
    lib.ob_server_stats.argtypes = [vp, C.POINTER(ServerSummary)]
    lib.ob_server_drain.argtypes = [vp, C.c_double]
    lib.ob_work_units.argtypes = [C.c_uint64, C.c_uint64, C.c_int32]
    lib.ob_work_units.restype = C.c_double
    cp = C.c_char_p
    lib.ob_checkpoint_write.argtypes = [cp, C.c_uint64, cp, C.c_uint64, C.c_uint64] + [_dp] * 10
    lib.ob_checkpoint_info.argtypes = [cp, _u64p, _u64p, _u64p]
    lib.ob_checkpoint_read.argtypes = [cp, C.c_char_p, C.c_uint64, C.c_uint64] + [_dp] * 10
    lib.ob_system_write_checkpoint.argtypes = [vp, cp, C.c_uint64, cp, C.c_uint64]
    lib.ob_system_read_checkpoint.argtypes = [vp, cp, _u64p, C.c_char_p, C.c_uint64, _u64p]
    lib.ob_trajectory_create.argtypes = [cp, C.c_uint64, _dp, C.c_double, C.c_int32,
                                         C.POINTER(vp)]
    lib.ob_trajectory_create_for_system.argtypes = [cp, vp, C.c_double, C.c_int32,
                                                    C.POINTER(vp)]
    lib.ob_trajectory_write_frame.argtypes = [vp, C.c_uint64, C.c_double] + [_dp] * 6
    lib.ob_trajectory_write_system_frame.argtypes = [vp, C.c_uint64, C.c_double]
    lib.ob_trajectory_flush.argtypes = [vp]
    lib.ob_trajectory_frames.argtypes = [vp, _u64p]
    lib.ob_trajectory_close.argtypes = [vp]
    # Every unsigned 64-bit argument (counts, steps, step indices, job ids)
    # refuses a value it cannot hold instead of wrapping it: -1 steps would
    # otherwise become 2^64 - 1 of them.
    for fn in list(vars(lib).values()):
        if isinstance(fn, C._CFuncPtr) and fn.argtypes:
            fn.argtypes = [_Unsigned64 if t is C.c_uint64 else t for t in fn.argtypes]
    _lib = lib
    return lib


def _count(value, what: str = "count") -> int:
    """An integer a uint64_t can hold: a count, a number of steps, a step index."""
    v = operator.index(value)
    if not 0 <= v < 1 << 64:
        raise OrreryError(ERROR_INVALID_ARGUMENT, f"{what} must be in [0, 2^64), not {v}")
    return v


class _Unsigned64(C.c_uint64):
    """A uint64_t argument that accepts only integers in [0, 2^64); ctypes
    reports a refused one as an ArgumentError."""

    @classmethod
    def from_param(cls, value):
        if isinstance(value, C.c_uint64):
            return value
        return C.c_uint64(_count(value))


def _check(rc: int) -> None:
    if rc != OK:
        raise OrreryError(rc, load_library().ob_last_error().decode())


def version() -> str:
    return load_library().ob_version().decode()


def device_count() -> int:
    n = C.c_int(0)
    _check(load_library().ob_device_count(C.byref(n)))
    return n.value


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def make_params(kind=SOLVER_DIRECT, precision="fp32", softening=0.0, opening_angle=0.5,
                leaf_capacity=32, quadrupole=False) -> SolverParams:
    prec = _PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    eps = float(softening)
    # core::Softening keeps the square, formed as length * length.
    return SolverParams(kind, prec, eps * eps, float(opening_angle), int(leaf_capacity),
                        1 if quadrupole else 0, 0)


class _Solver:
    """Common body of the two ForceSolver counterparts."""

    _name = ""

    def __init__(self, params: SolverParams):
        lib = load_library()
        handle = C.c_void_p()
        _check(lib.ob_solver_create(C.byref(params), C.byref(handle)))
        self._handle = handle
        self._lib = lib

    @classmethod
    def _try(cls, params: SolverParams):
        try:
            return cls(params)
        except OrreryError as e:
            if e.code == ERROR_NO_DEVICE:
                return None
            raise

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.ob_solver_destroy(h)
            self._handle = None

    def name(self) -> str:
        return self._name

    def params(self) -> SolverParams:
        p = SolverParams()
        _check(self._lib.ob_solver_get_params(self._handle, C.byref(p)))
        return p

    def softening(self) -> float:
        """The softening length (the square root of the stored square)."""
        return float(np.sqrt(self.params().softening_squared))

    def evaluate(self, positions, masses, accelerations=None) -> np.ndarray:
        """ForceSolver::evaluate: positions (3, N) or (N, 3) FP64, masses (N,).

        Writes into ``accelerations`` (three arrays x, y, z) when given --
        directly, without a copy, when they are contiguous FP64 of length N, in
        which case nothing is returned -- and otherwise returns the
        accelerations as an (N, 3) array."""
        x, y, z = _split_xyz(positions)
        m = _f64(masses)
        n = len(m)
        direct = accelerations is not None and all(
            isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
            and a.shape == (n,) for a in accelerations)
        out = list(accelerations) if direct else [np.empty(n) for _ in range(3)]
        _check(self._lib.ob_solver_evaluate(self._handle, n, _ptr(x), _ptr(y), _ptr(z), _ptr(m),
                                            _ptr(out[0]), _ptr(out[1]), _ptr(out[2])))
        if accelerations is not None and not direct:
            for k in range(3):
                accelerations[k][...] = out[k]
        if direct:
            return None
        return np.stack(out, axis=1)

    def evaluate_device(self, n, x, y, z, m, ax, ay, az, stream=0) -> None:
        """Device-pointer form (integers or objects with ``data_ptr()``)."""
        ptrs = [p.data_ptr() if hasattr(p, "data_ptr") else int(p)
                for p in (x, y, z, m, ax, ay, az)]
        _check(self._lib.ob_solver_evaluate_device(self._handle, _count(n, "n"), *ptrs,
                                                   stream or None))

    def interaction_count(self) -> InteractionCount:
        c = Counts()
        _check(self._lib.ob_solver_counts(self._handle, C.byref(c)))
        return InteractionCount(c.evaluations, c.particle_particle, c.particle_cell)

    def reset_interaction_count(self) -> None:
        _check(self._lib.ob_solver_reset_counts(self._handle))

    def set_shape(self, n: int, shape) -> None:
        """Fixes the direct kernel shape (threads, targets_per_thread, split[, groups])
        for n; groups defaults to 1."""
        if isinstance(shape, DirectShape):
            s = shape
        else:
            t = tuple(shape)
            s = DirectShape(*(t + (1,) * (4 - len(t))))
        _check(self._lib.ob_solver_set_direct_shape(self._handle, _count(n, "n"), C.byref(s)))

    def autotune(self, n: int):
        """Times every direct kernel shape for n particles; keeps and returns the best."""
        s = DirectShape()
        ms = C.c_double()
        _check(self._lib.ob_solver_autotune(self._handle, _count(n, "n"), C.byref(s), C.byref(ms)))
        return (s.threads, s.targets_per_thread, s.split, s.groups), ms.value

    def timings(self) -> dict:
        t = Timings()
        _check(self._lib.ob_solver_timings(self._handle, C.byref(t)))
        return {k: getattr(t, k) for k, _ in Timings._fields_}


class B200DirectSolver(_Solver):
    """Direct O(N^2) solver (the reference's DirectSolver / CudaDirectSolver)."""

    _name = "b200-direct"

    def __init__(self, softening: float = 0.0, precision: str = "fp32"):
        super().__init__(make_params(SOLVER_DIRECT, precision, softening))

    @classmethod
    def try_create(cls, softening: float = 0.0, precision: str = "fp32"):
        try:
            return cls(softening, precision)
        except OrreryError as e:
            if e.code == ERROR_NO_DEVICE:
                return None
            raise


class B200TreeSolver(_Solver):
    """Barnes-Hut solver (the reference's BarnesHutSolver / CudaTreeSolver).

    ``precision="fp32"`` computes FP32 forces on FP64 state; ``"fp64"`` is the
    parity mode, whose forces equal BarnesHutSolver's (scalar leaf kernel) bit
    for bit."""

    _name = "b200-tree"

    def __init__(self, softening: float = 0.0, opening_angle: float = 0.5,
                 leaf_capacity: int = 32, quadrupole: bool = False, precision: str = "fp32"):
        super().__init__(make_params(SOLVER_TREE, precision, softening, opening_angle,
                                     leaf_capacity, quadrupole))

    def tree_stats(self):
        """(node count, leaf count, depth) of the last tree."""
        nodes, leaves, depth = C.c_uint64(), C.c_uint64(), C.c_uint32()
        _check(self._lib.ob_tree_stats(self._handle, C.byref(nodes), C.byref(leaves),
                                       C.byref(depth)))
        return nodes.value, leaves.value, depth.value

    def tree(self):
        """The last octree: reals (n, 5) mass, com xyz, r2; idx (n, 3) next,
        first, count; quads (n, 6) or None; leaf count; depth."""
        nodes, leaves, depth = self.tree_stats()
        reals = np.zeros((nodes, 5))
        idx = np.zeros((nodes, 3), np.uint64)
        quad = bool(self.params().quadrupole)
        quads = np.zeros((nodes, 6)) if quad else None
        u64 = C.POINTER(C.c_uint64)
        _check(self._lib.ob_tree_copy(self._handle, _ptr(reals), idx.ctypes.data_as(u64),
                                      _ptr(quads) if quad else None))
        return reals, idx, quads, leaves, depth

    def order(self, n: int):
        """(codes uint64, indices, cube origin, cube size) of the last ordering."""
        codes = np.zeros(n, np.uint64)
        idx = np.zeros(n, np.uint32)
        origin = np.zeros(3)
        size = C.c_double()
        _check(self._lib.ob_tree_copy_order(
            self._handle, codes.ctypes.data_as(C.POINTER(C.c_uint64)),
            idx.ctypes.data_as(C.POINTER(C.c_uint32)), _ptr(origin), C.byref(size)))
        return codes, idx, origin, size.value

    @classmethod
    def try_create(cls, softening: float = 0.0, opening_angle: float = 0.5,
                   leaf_capacity: int = 32, quadrupole: bool = False, precision: str = "fp32"):
        try:
            return cls(softening, opening_angle, leaf_capacity, quadrupole, precision)
        except OrreryError as e:
            if e.code == ERROR_NO_DEVICE:
                return None
            raise


def direct_shapes(precision: str = "fp32"):
    """Every (threads, targets_per_thread, split, groups) shape of a direct kernel."""
    lib = load_library()
    count = C.c_int32()
    _check(lib.ob_direct_shapes(_PRECISIONS[precision], None, 0, C.byref(count)))
    arr = (DirectShape * count.value)()
    _check(lib.ob_direct_shapes(_PRECISIONS[precision], arr, count.value, C.byref(count)))
    return [(s.threads, s.targets_per_thread, s.split, s.groups) for s in arr]


# The reference's ParticleData names (python/src/core_bindings.cpp:253-300) and
# the keys this package uses for the same arrays.
_PARTICLE_NAMES = {"position_x": "x", "position_y": "y", "position_z": "z",
                   "velocity_x": "vx", "velocity_y": "vy", "velocity_z": "vz",
                   "acceleration_x": "ax", "acceleration_y": "ay", "acceleration_z": "az",
                   "mass": "m"}


def _state_of(state) -> dict:
    """A state given as a dict keyed x ... m, or as the reference's
    ParticleData (anything with position_x ... mass), as a dict keyed x ... m."""
    if hasattr(state, "keys") and "m" in state:
        return state
    if all(hasattr(state, name) for name in _PARTICLE_NAMES if not name.startswith("acc")):
        return {key: getattr(state, name) for name, key in _PARTICLE_NAMES.items()
                if hasattr(state, name)}
    raise OrreryError(ERROR_INVALID_ARGUMENT,
                      "a state is a dict of x y z vx vy vz m or a ParticleData")


def _split_xyz(positions):
    if isinstance(positions, (tuple, list)) and len(positions) == 3 and \
            all(np.ndim(a) == 1 for a in positions):
        return tuple(_f64(a) for a in positions)
    p = np.asarray(positions, dtype=np.float64)
    if p.ndim == 2 and p.shape[0] == 3 and p.shape[1] != 3:
        return tuple(_f64(p[k]) for k in range(3))
    if p.ndim == 2 and p.shape[1] == 3:
        return tuple(_f64(p[:, k]) for k in range(3))
    if p.ndim == 2 and p.shape == (3, 3):
        return tuple(_f64(p[:, k]) for k in range(3))
    raise ValueError("positions must be (N, 3), (3, N) or a tuple of three arrays")


class DeviceSystem:
    """A particle system resident in HBM, integrated on the device.

    ``step(dt, steps, integrator)`` advances with velocity Verlet or Yoshida-4
    (src/integrators/velocity_verlet.cpp:59-72, yoshida4.cpp:45-59); one step is
    a replayed CUDA graph and no state crosses to the host between steps."""

    def __init__(self, n: int, softening: float = 0.0, kind: int = SOLVER_DIRECT,
                 precision: str = "fp32", opening_angle: float = 0.5, leaf_capacity: int = 32,
                 quadrupole: bool = False):
        lib = load_library()
        handle = C.c_void_p()
        params = make_params(kind, precision, softening, opening_angle, leaf_capacity,
                             quadrupole)
        _check(lib.ob_system_create(C.byref(params), _count(n, "n"), C.byref(handle)))
        self._lib = lib
        self._handle = handle
        self.n = _count(n, "n")

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.ob_system_destroy(h)
            self._handle = None

    def set_state(self, x, y, z, vx=None, vy=None, vz=None, m=None) -> None:
        arrs = [_f64(a) if a is not None else None for a in (x, y, z, vx, vy, vz, m)]
        _check(self._lib.ob_system_set_state(self._handle, *(_ptr(a) for a in arrs)))

    def set_accelerations(self, ax, ay, az) -> None:
        arrs = [_f64(a) for a in (ax, ay, az)]
        _check(self._lib.ob_system_set_accelerations(self._handle, *(_ptr(a) for a in arrs)))

    def state(self) -> dict:
        out = {k: np.empty(self.n) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
        _check(self._lib.ob_system_get_state(self._handle, *(_ptr(out[k]) for k in (
            "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"))))
        return out

    def step(self, dt: float, steps: int = 1, integrator: str = "vv") -> None:
        _check(self._lib.ob_system_step(self._handle, _INTEGRATORS[integrator], float(dt),
                                        _count(steps, "steps")))

    def step_host(self, state: dict, dt: float, steps: int = 1, integrator: str = "vv") -> None:
        """Integrator::step over host arrays: state holds x y z vx vy vz ax ay az m
        (contiguous FP64, updated in place)."""
        keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")
        for k in keys:
            a = state[k]
            if a.dtype != np.float64 or not a.flags.c_contiguous or len(a) != self.n:
                raise OrreryError(ERROR_INVALID_ARGUMENT, f"{k} must be contiguous FP64 of n")
        _check(self._lib.ob_system_step_host(self._handle, _INTEGRATORS[integrator], float(dt),
                                             _count(steps, "steps"),
                                             *(_ptr(state[k]) for k in keys)))

    def step_async(self, dt: float, steps: int = 1, integrator: str = "vv") -> None:
        _check(self._lib.ob_system_step_async(self._handle, _INTEGRATORS[integrator], float(dt),
                                              _count(steps, "steps")))

    def synchronize(self) -> None:
        _check(self._lib.ob_system_synchronize(self._handle))

    def write_checkpoint(self, path, step: int, configuration: str = "") -> None:
        """An ORRERYCK v1 checkpoint of the device state after `step` steps
        (sim::write_checkpoint); `configuration` is the reference's
        configuration text, stored as is."""
        text = configuration.encode()
        _check(self._lib.ob_system_write_checkpoint(self._handle, os.fsencode(path),
                                                    _count(step, "step"), text, len(text)))

    def read_checkpoint(self, path):
        """Restores the state (carried accelerations included) from an ORRERYCK
        v1 checkpoint of this size; returns (step, configuration text)."""
        step, n, size = (C.c_uint64() for _ in range(3))
        _check(self._lib.ob_checkpoint_info(os.fsencode(path), C.byref(step), C.byref(n),
                                            C.byref(size)))
        buf = C.create_string_buffer(max(1, size.value))
        got = C.c_uint64()
        _check(self._lib.ob_system_read_checkpoint(self._handle, os.fsencode(path),
                                                   C.byref(step), buf, size.value,
                                                   C.byref(got)))
        return step.value, buf.raw[:got.value].decode()

    def energy(self):
        ke, pe = C.c_double(), C.c_double()
        _check(self._lib.ob_system_energy(self._handle, C.byref(ke), C.byref(pe)))
        return ke.value, pe.value

    def diagnostics(self) -> dict:
        """core::measure_diagnostics of the state: kinetic_energy,
        potential_energy, linear_momentum (3), angular_momentum (3)."""
        d = DiagnosticsRecord()
        _check(self._lib.ob_system_diagnostics(self._handle, C.byref(d)))
        return {"kinetic_energy": d.kinetic_energy, "potential_energy": d.potential_energy,
                "linear_momentum": np.array(d.linear_momentum[:]),
                "angular_momentum": np.array(d.angular_momentum[:])}

    def snapshot(self) -> dict:
        """The whole state on the host: x y z vx vy vz ax ay az and m."""
        keys = ("m", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
        out = {k: np.empty(self.n) for k in keys}
        _check(self._lib.ob_system_snapshot(self._handle, *(_ptr(out[k]) for k in keys)))
        return out

    def kinetic_energy(self) -> float:
        ke = C.c_double()
        _check(self._lib.ob_system_energy(self._handle, C.byref(ke), None))
        return ke.value

    def interaction_count(self) -> InteractionCount:
        c = Counts()
        _check(self._lib.ob_system_counts(self._handle, C.byref(c)))
        return InteractionCount(c.evaluations, c.particle_particle, c.particle_cell)

    def autotune(self):
        """Times every direct kernel shape at this system's size and keeps the best."""
        s = DirectShape()
        ms = C.c_double()
        _check(self._lib.ob_system_autotune(self._handle, C.byref(s), C.byref(ms)))
        return (s.threads, s.targets_per_thread, s.split, s.groups), ms.value

    def stream(self) -> int:
        """The cudaStream_t (as an integer) the system enqueues its work on."""
        s = C.c_void_p()
        _check(self._lib.ob_system_stream(self._handle, C.byref(s)))
        return s.value or 0

    def profile(self, steps: int) -> None:
        """Record per-phase events for the next ``steps`` steps."""
        _check(self._lib.ob_system_profile(self._handle, _count(steps, "steps")))

    def phase_times(self):
        """Per-evaluation average phase times (ms) over the profiled steps."""
        t = Timings()
        n = C.c_uint32()
        _check(self._lib.ob_system_phase_times(self._handle, C.byref(t), C.byref(n)))
        return {k: getattr(t, k) for k, _ in Timings._fields_}, n.value

    def set_fused_steps(self, enable: bool = True) -> bool:
        """Allows (default) or forbids whole steps of a small FP32-direct system
        in one launch; returns whether the next velocity-Verlet step uses it."""
        active = C.c_int32()
        _check(self._lib.ob_system_set_fused_steps(self._handle, 1 if enable else 0,
                                                   C.byref(active)))
        return bool(active.value)

    def step_kernels(self, dt: float, integrator: str = "vv") -> int:
        """Kernel launches one step call makes (a captured step's kernels, or one
        launch for the fused small-system path, whatever the step count)."""
        k = C.c_uint32()
        _check(self._lib.ob_system_step_kernels(self._handle, _INTEGRATORS[integrator],
                                                float(dt), C.byref(k)))
        return k.value


def probe_fp32():
    """Measured (FFMA lane ops/s, SFU rsqrt lane ops/s) of the current device."""
    a, b = C.c_double(), C.c_double()
    _check(load_library().ob_probe_fp32(C.byref(a), C.byref(b)))
    return a.value, b.value


def probe_fp64() -> float:
    """Measured FP64 FMA lane operations per second of the current device."""
    r = C.c_double()
    _check(load_library().ob_probe_fp64(C.byref(r)))
    return r.value


def probe_fp32x2() -> float:
    """Measured FMAs per second issued as packed FP32x2 instructions."""
    a = C.c_double()
    _check(load_library().ob_probe_fp32x2(C.byref(a)))
    return a.value


class DeviceBatch:
    """Many independent systems of uneven size, each with its own softening,
    evaluated in one persistent launch and stepped together (precision form:
    split FP32 pair arithmetic with FP64 accumulation)."""

    KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")

    def __init__(self, counts, softenings):
        lib = load_library()
        counts = np.ascontiguousarray(counts, dtype=np.uint64)
        eps = np.asarray(softenings, dtype=np.float64)
        eps2 = np.ascontiguousarray(eps * eps)
        handle = C.c_void_p()
        _check(lib.ob_batch_create(len(counts), counts.ctypes.data_as(C.POINTER(C.c_uint64)),
                                   _ptr(eps2), C.byref(handle)))
        self._lib = lib
        self._handle = handle
        self.counts = [int(c) for c in counts]

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.ob_batch_destroy(h)
            self._handle = None

    def set_state(self, system, x, y, z, vx=None, vy=None, vz=None, m=None) -> None:
        arrs = [_f64(a) if a is not None else None for a in (x, y, z, vx, vy, vz, m)]
        _check(self._lib.ob_batch_set_state(self._handle, int(system),
                                            *(_ptr(a) for a in arrs)))

    def refresh(self) -> None:
        _check(self._lib.ob_batch_refresh(self._handle))

    def state(self, system) -> dict:
        n = self.counts[system]
        out = {k: np.empty(n) for k in self.KEYS}
        _check(self._lib.ob_batch_get_state(self._handle, int(system),
                                            *(_ptr(out[k]) for k in self.KEYS)))
        return out

    def step(self, dt: float, steps: int = 1, integrator: str = "yoshida4") -> None:
        _check(self._lib.ob_batch_step(self._handle, _INTEGRATORS[integrator], float(dt),
                                       _count(steps, "steps")))

    def step_async(self, dt: float, steps: int = 1, integrator: str = "yoshida4") -> None:
        _check(self._lib.ob_batch_step_async(self._handle, _INTEGRATORS[integrator], float(dt),
                                             _count(steps, "steps")))

    def synchronize(self) -> None:
        _check(self._lib.ob_batch_synchronize(self._handle))

    def energy(self, system):
        ke, pe = C.c_double(), C.c_double()
        _check(self._lib.ob_batch_energy(self._handle, int(system), C.byref(ke), C.byref(pe)))
        return ke.value, pe.value

    def autotune(self):
        s = BatchShape()
        ms = C.c_double()
        _check(self._lib.ob_batch_autotune(self._handle, C.byref(s), C.byref(ms)))
        return (s.threads, s.targets_per_thread, s.chunk_tiles, s.groups), ms.value

    def set_shape(self, threads, targets_per_thread, chunk_tiles, groups=1) -> None:
        s = BatchShape(threads, targets_per_thread, chunk_tiles, groups)
        _check(self._lib.ob_batch_set_shape(self._handle, C.byref(s)))

    def stats(self):
        pairs, evals, items = C.c_uint64(), C.c_uint64(), C.c_uint32()
        _check(self._lib.ob_batch_stats(self._handle, C.byref(pairs), C.byref(evals),
                                        C.byref(items)))
        return pairs.value, evals.value, items.value

    def stream(self) -> int:
        s = C.c_void_p()
        _check(self._lib.ob_batch_stream(self._handle, C.byref(s)))
        return s.value or 0


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED, JOB_REJECTED = range(6)


class Server:
    """The persistent serving loop (continuous batching, HBM-budget admission).

    ``fake=True`` runs the same scheduler with no GPU: each step takes the time
    a cost model gives (direct: pairs / fake_direct_gint_s; tree: N x
    fake_tree_ns_per_particle)."""

    def __init__(self, hbm_budget_bytes: int, direct_pairs_cap: int = 0,
                 direct_arena_particles: int = 0, max_tree_jobs: int = 1, fake: bool = False,
                 fake_direct_gint_s: float = 800.0, fake_tree_ns_per_particle: float = 12.0,
                 max_job_work: float = 0.0, max_running_work: float = 0.0):
        lib = load_library()
        cfg = ServerConfig(int(hbm_budget_bytes), int(direct_pairs_cap),
                           int(direct_arena_particles), int(max_tree_jobs), 1 if fake else 0,
                           float(fake_direct_gint_s), float(fake_tree_ns_per_particle),
                           float(max_job_work), float(max_running_work))
        handle = C.c_void_p()
        _check(lib.ob_server_create(C.byref(cfg), C.byref(handle)))
        self._lib = lib
        self._handle = handle
        self._sizes = {}

    def close(self) -> None:
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.ob_server_destroy(h)
            self._handle = None

    def __del__(self):
        self.close()

    def submit(self, state: dict, steps: int, dt: float, softening: float, kind: str = "direct",
               integrator: str = "yoshida4", opening_angle: float = 0.5,
               leaf_capacity: int = 32, quadrupole: bool = True) -> int:
        solvers = {"direct": SOLVER_DIRECT, "tree": SOLVER_TREE}
        if kind not in solvers:
            raise OrreryError(ERROR_INVALID_ARGUMENT,
                              f"unknown job kind {kind!r} (expected 'direct' or 'tree')")
        if integrator not in _INTEGRATORS:
            raise OrreryError(ERROR_INVALID_ARGUMENT, f"unknown integrator {integrator!r}")
        state = _state_of(state)
        n = len(state["m"])
        spec = JobSpec(solvers[kind],
                       _INTEGRATORS[integrator], n, _count(steps, "steps"), float(dt),
                       float(softening) * float(softening), float(opening_angle),
                       int(leaf_capacity), 1 if quadrupole else 0, 0)
        arrs = [_f64(state[k]) if state.get(k) is not None else None
                for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        job = C.c_uint64()
        _check(self._lib.ob_server_submit(self._handle, C.byref(spec),
                                          *(_ptr(a) for a in arrs), C.byref(job)))
        self._sizes[job.value] = n
        return job.value

    def wait(self, job: int, timeout: float = 600.0, outputs: bool = True):
        """(report dict, final state dict or None)."""
        n = self._sizes.get(job, 0)
        outputs = outputs and n > 0
        keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
        out = {k: np.empty(n) for k in keys} if outputs else None
        rep = JobReport()
        ptrs = [(_ptr(out[k]) if outputs else None) for k in keys]
        _check(self._lib.ob_server_wait(self._handle, int(job), float(timeout), C.byref(rep),
                                        *ptrs))
        report = {k: getattr(rep, k) for k, _ in JobReport._fields_ if k != "reserved"}
        return report, (out if outputs and rep.status == JOB_DONE else None)

    def cancel(self, job: int) -> None:
        _check(self._lib.ob_server_cancel(self._handle, int(job)))

    def stats(self) -> dict:
        s = ServerSummary()
        _check(self._lib.ob_server_stats(self._handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerSummary._fields_}

    def drain(self, timeout: float = 600.0) -> None:
        _check(self._lib.ob_server_drain(self._handle, float(timeout)))


_CHECKPOINT_ARRAYS = ("m", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def write_checkpoint(path, step: int, state: dict, configuration: str = "") -> None:
    """sim::write_checkpoint (include/orrery/sim/checkpoint.hpp:85) from host
    arrays: `state` holds m x y z vx vy vz ax ay az (FP64, equal lengths)."""
    arrs = [_f64(state[k]) for k in _CHECKPOINT_ARRAYS]
    n = len(arrs[0])
    if any(len(a) != n for a in arrs):
        raise OrreryError(ERROR_INVALID_ARGUMENT, "every state array needs the same length")
    text = configuration.encode()
    lib = load_library()
    _check(lib.ob_checkpoint_write(os.fsencode(path), _count(step, "step"), text, len(text), n,
                                   *(_ptr(a) for a in arrs)))


def checkpoint_info(path) -> dict:
    """The header of an ORRERYCK checkpoint: step, particle count, configuration length."""
    lib = load_library()
    step, n, size = (C.c_uint64() for _ in range(3))
    _check(lib.ob_checkpoint_info(os.fsencode(path), C.byref(step), C.byref(n), C.byref(size)))
    return {"step": step.value, "n": n.value, "configuration_bytes": size.value}


def read_checkpoint(path) -> dict:
    """sim::read_checkpoint (include/orrery/sim/checkpoint.hpp:94): the step,
    the configuration text and the ten state arrays, checked against the
    file's checksum."""
    info = checkpoint_info(path)
    n = info["n"]
    out = {k: np.empty(n) for k in _CHECKPOINT_ARRAYS}
    buf = C.create_string_buffer(max(1, info["configuration_bytes"]))
    lib = load_library()
    _check(lib.ob_checkpoint_read(os.fsencode(path), buf, info["configuration_bytes"], n,
                                  *(_ptr(out[k]) for k in _CHECKPOINT_ARRAYS)))
    out["step"] = info["step"]
    out["configuration"] = buf.raw[:info["configuration_bytes"]].decode()
    return out


class Trajectory:
    """sim::TrajectoryWriter (include/orrery/sim/trajectory.hpp:112-146): an
    ORRERYTJ v1 file. Over host arrays (``masses`` given), or bound to a
    DeviceSystem (``system`` given), whose frames are snapshots taken on the
    device between steps and written by a background thread."""

    def __init__(self, path, timestep: float, masses=None, system=None,
                 with_velocities: bool = False):
        lib = load_library()
        handle = C.c_void_p()
        if system is not None:
            _check(lib.ob_trajectory_create_for_system(os.fsencode(path), system._handle,
                                                       float(timestep), int(with_velocities),
                                                       C.byref(handle)))
            self.n = system.n
        else:
            m = _f64(masses)
            _check(lib.ob_trajectory_create(os.fsencode(path), len(m), _ptr(m), float(timestep),
                                            int(with_velocities), C.byref(handle)))
            self.n = len(m)
        self._lib = lib
        self._handle = handle
        self._system = system  # kept alive while the trajectory is open
        self.with_velocities = bool(with_velocities)

    def write_frame(self, step: int, time: float, state: dict = None) -> None:
        """A frame from host arrays (x y z, and vx vy vz when the file carries
        them), or, with no `state`, a snapshot of the bound system."""
        if state is None:
            _check(self._lib.ob_trajectory_write_system_frame(self._handle, _count(step, "step"),
                                                              float(time)))
            return
        keys = ("x", "y", "z", "vx", "vy", "vz") if self.with_velocities else ("x", "y", "z")
        arrs = [_f64(state[k]) for k in keys] + [None] * (6 - len(keys))
        _check(self._lib.ob_trajectory_write_frame(self._handle, _count(step, "step"), float(time),
                                                   *(_ptr(a) for a in arrs)))

    def flush(self) -> None:
        _check(self._lib.ob_trajectory_flush(self._handle))

    @property
    def frames(self) -> int:
        f = C.c_uint64()
        _check(self._lib.ob_trajectory_frames(self._handle, C.byref(f)))
        return f.value

    def close(self) -> None:
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._handle = None
            _check(self._lib.ob_trajectory_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.ob_trajectory_close(h)
            self._handle = None


def work_units(count: int, steps: int, solver: str) -> float:
    """The reference service's cost of a run (service/orrery_service/limits.py:82-111),
    as the server's admission counts it: count^2 * steps for "direct",
    count * log2(count) * steps for the tree ("barnes-hut" or "tree")."""
    kind = SOLVER_DIRECT if solver == "direct" else SOLVER_TREE
    return load_library().ob_work_units(_count(count, "count"), _count(steps, "steps"), kind)


_PARTICLE_ARRAYS = ("position_x", "position_y", "position_z", "mass",
                    "acceleration_x", "acceleration_y", "acceleration_z")


def compute_accelerations(positions, masses, softening: float = 0.0, solver: str = "direct",
                          precision: str = None, opening_angle: float = 0.5,
                          leaf_capacity: int = 32, quadrupole: bool = False):
    """One force evaluation, the counterpart of the reference's Python
    ``orrery.compute_accelerations`` (python/src/sim_bindings.cpp:383-410).

    Two forms:

    * ``compute_accelerations(positions, masses, ...)``: positions (N, 3) or
      (3, N) and masses (N,); returns the (N, 3) accelerations. Precision
      defaults to "fp32".
    * ``compute_accelerations(configuration, particles)``, the reference's own
      call: ``configuration.solver`` supplies the kind ("direct" or
      "barnes-hut"; the reference's "sycl-direct" and "sycl-tree" name the
      same algorithms on a device), softening, opening angle, leaf capacity
      and quadrupole flag; ``particles`` is the reference's ParticleData (or
      anything with its position_x ... mass and acceleration_x ... arrays).
      The accelerations are written into the particles in place and the
      InteractionCount is returned. Precision defaults to "fp64", whose forces
      equal the reference's DirectSolver and BarnesHutSolver (scalar kernels)
      bit for bit; the other settings of the configuration are not read.
    """
    if hasattr(positions, "solver") and all(hasattr(masses, k) for k in _PARTICLE_ARRAYS):
        settings, particles = positions.solver, masses
        kind = str(settings.kind)
        precision = precision or "fp64"
        if kind in ("direct", "sycl-direct"):
            s = B200DirectSolver(float(settings.softening), precision)
        elif kind in ("barnes-hut", "sycl-tree"):
            s = B200TreeSolver(float(settings.softening), float(settings.opening_angle),
                               int(settings.leaf_capacity), bool(settings.quadrupole),
                               precision)
        else:
            raise OrreryError(ERROR_INVALID_ARGUMENT, f"unknown solver kind {kind!r}")
        xyz = [np.asarray(getattr(particles, k)) for k in _PARTICLE_ARRAYS[:3]]
        s.evaluate(xyz, np.asarray(particles.mass),
                   [np.asarray(getattr(particles, k)) for k in _PARTICLE_ARRAYS[4:]])
        return s.interaction_count()
    precision = precision or "fp32"
    if solver == "direct":
        s = B200DirectSolver(softening, precision)
    elif solver in ("tree", "barnes-hut"):
        s = B200TreeSolver(softening, opening_angle, leaf_capacity, quadrupole, precision)
    else:
        raise ValueError(f"unknown solver {solver!r}")
    return s.evaluate(positions, masses)


from .simulation import (DeviceArrayView, Diagnostics, DiagnosticsLog, FileOutput,  # noqa: E402,F401
                         Particles, Simulation, Vec3, device_arrays)
