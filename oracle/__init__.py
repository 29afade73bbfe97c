"""Python access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two libraries, both built by ``oracle/Makefile``:

* ``restatement`` -- ``_lib/liboracle.so``, the plain-C restatement of the
  reference's FP64 path (oracle.c). Always available once built.
* ``reference`` -- ``_ref/libref_orrery.so``, the reference's own CPU sources
  compiled where they lie, behind a small C shim (ref_shim.cpp). Present only
  where it was built (it travels with the repository snapshot as a built file).
* ``reference CUDA`` -- ``_ref/libref_orrery_cuda.so``, the same plus the
  reference's CUDA solvers (its .cu kernels compiled for sm_100a), behind
  ref_cuda_shim.cpp: the reference's GPU path, timed beside this backend's.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package. The product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_PATH = os.path.join(HERE, "_lib", "liboracle.so")
REFERENCE_PATH = os.path.join(HERE, "_ref", "libref_orrery.so")
REFERENCE_CUDA_PATH = os.path.join(HERE, "_ref", "libref_orrery_cuda.so")
REFERENCE_CUDA_SINGLE_PATH = os.path.join(HERE, "_ref", "libref_orrery_cuda_single.so")
REFERENCE_ROOT_RECORD = os.path.join(HERE, "_ref", "reference_root.txt")

_dp = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)


def _d(a):
    return a.ctypes.data_as(_dp)


def _u(a):
    return a.ctypes.data_as(_u64p)


def build(reference_root: str | None = None, with_reference: bool = True) -> None:
    """Compile the restatement, and -- given the reference's checkout, by argument
    or by the ORRERY_REFERENCE_ROOT environment variable -- the reference's own
    libraries and the adapter test driver. Without a checkout the reference
    libraries are left as they are (built ones travel with the repository)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    root = reference_root or os.environ.get("ORRERY_REFERENCE_ROOT")
    if not with_reference or not root:
        return
    if not os.path.isdir(os.path.join(root, "src", "solvers")):
        raise FileNotFoundError(f"{root} holds no reference checkout (src/solvers is missing)")
    subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", "ref_cuda", "ref_cuda_single",
                    "ref_adapter", f"REF={root}"], check=True)
    with open(REFERENCE_ROOT_RECORD, "w") as fh:
        fh.write(os.path.abspath(root))


def reference_root() -> str | None:
    """The reference checkout: ORRERY_REFERENCE_ROOT, else the one the last
    build() used (recorded beside the libraries it built); None when neither
    names an existing directory."""
    root = os.environ.get("ORRERY_REFERENCE_ROOT")
    if not root and os.path.exists(REFERENCE_ROOT_RECORD):
        with open(REFERENCE_ROOT_RECORD) as fh:
            root = fh.read().strip()
    return root if root and os.path.isdir(root) else None


class Counts(C.Structure):
    _fields_ = [("evaluations", C.c_uint64), ("particle_particle", C.c_uint64),
                ("particle_cell", C.c_uint64)]


class _Node(C.Structure):
    _fields_ = [("mass", C.c_double), ("com_x", C.c_double), ("com_y", C.c_double),
                ("com_z", C.c_double), ("acceptance_radius_squared", C.c_double),
                ("next", C.c_uint64), ("first_particle", C.c_uint64),
                ("particle_count", C.c_uint64)]


class _Tree(C.Structure):
    _fields_ = [("nodes", C.POINTER(_Node)), ("quadrupoles", C.POINTER(C.c_double)),
                ("node_count", C.c_size_t), ("capacity", C.c_size_t),
                ("leaf_count", C.c_size_t), ("depth", C.c_uint),
                ("opening_angle", C.c_double), ("leaf_capacity", C.c_uint64)]


class Tree:
    """An octree as arrays: reals (n, 5) = mass, com xyz, r2; idx (n, 3) = next, first, count."""

    def __init__(self, reals, idx, quads, leaf_count, depth):
        self.reals = reals
        self.idx = idx
        self.quads = quads
        self.leaf_count = int(leaf_count)
        self.depth = int(depth)

    @property
    def node_count(self) -> int:
        return int(self.reals.shape[0])


class Restatement:
    """ctypes binding of oracle.c."""

    def __init__(self, path: str = RESTATEMENT_PATH):
        if not os.path.exists(path):
            build(with_reference=False)
        lib = C.CDLL(path)
        self.lib = lib
        lib.oc_direct.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp,
                                  C.POINTER(Counts)]
        lib.oc_reference_acceleration.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_size_t,
                                                  C.c_double, _dp]
        lib.oc_bounding_cube.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, _dp]
        lib.oc_spread_bits.argtypes = [C.c_uint32]
        lib.oc_spread_bits.restype = C.c_uint64
        lib.oc_morton_code_grid.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        lib.oc_morton_code_grid.restype = C.c_uint64
        lib.oc_morton_code.argtypes = [C.c_double, C.c_double, C.c_double, _dp, C.c_double]
        lib.oc_morton_code.restype = C.c_uint64
        lib.oc_morton_octant.argtypes = [C.c_uint64, C.c_uint]
        lib.oc_morton_octant.restype = C.c_uint
        lib.oc_morton_order.argtypes = [C.c_size_t, _dp, _dp, _dp, _u64p, _u64p, _dp, _dp]
        lib.oc_tree_build.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, _u64p, _dp, C.c_double,
                                      C.c_double, C.c_uint64, C.c_int, C.POINTER(_Tree)]
        lib.oc_tree_free.argtypes = [C.POINTER(_Tree)]
        lib.oc_barnes_hut.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                      C.c_uint64, C.c_int, _dp, _dp, _dp, C.POINTER(Counts)]
        lib.oc_barnes_hut_targets.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double,
                                              C.c_double, C.c_uint64, C.c_int, C.c_size_t,
                                              _u64p, _dp, _u64p, _u64p]
        for name in ("oc_vv_step_direct", "oc_yoshida_step_direct", "oc_rk4_step_direct"):
            getattr(lib, name).argtypes = [C.c_size_t] + [_dp] * 10 + [C.c_double, C.c_double,
                                                                       C.POINTER(Counts)]
        lib.oc_yoshida_weights.argtypes = [_dp, _dp]
        lib.oc_kinetic_energy.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp]
        lib.oc_kinetic_energy.restype = C.c_double
        lib.oc_potential_energy.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double]
        lib.oc_potential_energy.restype = C.c_double

    # -- direct --------------------------------------------------------------
    def direct(self, x, y, z, m, softening):
        n = len(m)
        a = [np.zeros(n) for _ in range(3)]
        counts = Counts()
        self.lib.oc_direct(n, _d(x), _d(y), _d(z), _d(m), softening, _d(a[0]), _d(a[1]),
                           _d(a[2]), C.byref(counts))
        return np.stack(a, axis=1), counts

    def reference_acceleration(self, x, y, z, m, target, softening):
        out = np.zeros(3)
        self.lib.oc_reference_acceleration(len(m), _d(x), _d(y), _d(z), _d(m), target, softening,
                                           _d(out))
        return out

    def reference_accelerations(self, x, y, z, m, softening, targets=None):
        targets = range(len(m)) if targets is None else targets
        return np.array([self.reference_acceleration(x, y, z, m, int(t), softening)
                         for t in targets]).reshape(-1, 3)

    # -- Morton --------------------------------------------------------------
    def bounding_cube(self, x, y, z):
        origin = np.zeros(3)
        size = C.c_double()
        self.lib.oc_bounding_cube(len(x), _d(x), _d(y), _d(z), _d(origin), C.byref(size))
        return origin, size.value

    def spread_bits(self, v):
        return self.lib.oc_spread_bits(v)

    def morton_code_grid(self, gx, gy, gz):
        return self.lib.oc_morton_code_grid(gx, gy, gz)

    def morton_code(self, p, origin, size):
        origin = np.ascontiguousarray(origin, dtype=np.float64)
        return self.lib.oc_morton_code(p[0], p[1], p[2], _d(origin), size)

    def morton_octant(self, code, level):
        return self.lib.oc_morton_octant(code, level)

    def morton_order(self, x, y, z):
        n = len(x)
        codes = np.zeros(n, np.uint64)
        idx = np.zeros(n, np.uint64)
        origin = np.zeros(3)
        size = C.c_double()
        self.lib.oc_morton_order(n, _d(x), _d(y), _d(z), _u(codes), _u(idx), _d(origin),
                                 C.byref(size))
        return codes, idx, origin, size.value

    # -- tree ----------------------------------------------------------------
    def tree(self, x, y, z, m, opening_angle=0.5, leaf_capacity=32, quadrupole=False):
        """Morton-order the particles and build the octree; returns (Tree, codes, idx)."""
        codes, idx, origin, size = self.morton_order(x, y, z)
        ii = idx.astype(np.int64)
        sx, sy, sz, sm = (np.ascontiguousarray(a[ii]) for a in (x, y, z, m))
        t = _Tree()
        rc = self.lib.oc_tree_build(len(m), _d(sx), _d(sy), _d(sz), _d(sm), _u(codes),
                                    _d(origin), size, opening_angle, leaf_capacity,
                                    1 if quadrupole else 0, C.byref(t))
        if rc != 0:
            raise MemoryError("oracle tree build failed")
        n = t.node_count
        reals = np.zeros((n, 5))
        ind = np.zeros((n, 3), np.uint64)
        quads = np.zeros((n, 6)) if quadrupole else None
        if n:
            nodes = np.ctypeslib.as_array(C.cast(t.nodes, C.POINTER(C.c_uint8)),
                                          shape=(n * C.sizeof(_Node),))
            rec = np.frombuffer(nodes.tobytes(), dtype=np.dtype([
                ("r", np.float64, 5), ("i", np.uint64, 3)]))
            reals[:] = rec["r"]
            ind[:] = rec["i"]
            if quadrupole:
                quads[:] = np.ctypeslib.as_array(t.quadrupoles, shape=(n * 6,)).reshape(n, 6)
        tree = Tree(reals, ind, quads, t.leaf_count, t.depth)
        self.lib.oc_tree_free(C.byref(t))
        return tree, codes, idx

    def barnes_hut(self, x, y, z, m, softening, opening_angle=0.5, leaf_capacity=32,
                   quadrupole=False):
        n = len(m)
        a = [np.zeros(n) for _ in range(3)]
        counts = Counts()
        rc = self.lib.oc_barnes_hut(n, _d(x), _d(y), _d(z), _d(m), softening, opening_angle,
                                    leaf_capacity, 1 if quadrupole else 0, _d(a[0]), _d(a[1]),
                                    _d(a[2]), C.byref(counts))
        if rc != 0:
            raise MemoryError("oracle Barnes-Hut failed")
        return np.stack(a, axis=1), counts

    def barnes_hut_targets(self, x, y, z, m, softening, opening_angle, leaf_capacity,
                           quadrupole, targets):
        """Accelerations (k, 3), pair and cell counts of the listed targets only."""
        t = np.ascontiguousarray(targets, dtype=np.uint64)
        k = len(t)
        acc = np.zeros((k, 3))
        pairs = np.zeros(k, np.uint64)
        cells = np.zeros(k, np.uint64)
        rc = self.lib.oc_barnes_hut_targets(len(m), _d(x), _d(y), _d(z), _d(m), softening,
                                            opening_angle, leaf_capacity,
                                            1 if quadrupole else 0, k, _u(t), _d(acc),
                                            _u(pairs), _u(cells))
        if rc != 0:
            raise MemoryError("oracle Barnes-Hut failed")
        return acc, pairs, cells

    # -- integrators and energies -------------------------------------------
    def integrate_direct(self, state, m, softening, dt, steps, integrator="vv"):
        """Advance ``state`` (dict of x y z vx vy vz ax ay az arrays, copied) in place."""
        s = {k: np.ascontiguousarray(v, dtype=np.float64).copy() for k, v in state.items()}
        fn = {"yoshida4": self.lib.oc_yoshida_step_direct, "rk4": self.lib.oc_rk4_step_direct,
              "vv": self.lib.oc_vv_step_direct}[integrator]
        counts = Counts()
        for _ in range(steps):
            fn(len(m), *(_d(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")),
               _d(m), softening, dt, C.byref(counts))
        return s, counts

    def yoshida_weights(self):
        a, b = C.c_double(), C.c_double()
        self.lib.oc_yoshida_weights(C.byref(a), C.byref(b))
        return a.value, b.value

    def kinetic_energy(self, vx, vy, vz, m):
        return self.lib.oc_kinetic_energy(len(m), _d(vx), _d(vy), _d(vz), _d(m))

    def potential_energy(self, x, y, z, m, softening):
        return self.lib.oc_potential_energy(len(m), _d(x), _d(y), _d(z), _d(m), softening)


class Reference:
    """ctypes binding of the reference's own CPU code (libref_orrery.so)."""

    def __init__(self, path: str = REFERENCE_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        self.lib = lib
        lib.ref_default_worker_count.restype = C.c_uint
        lib.ref_plummer.argtypes = [C.c_size_t, C.c_double, C.c_double, C.c_uint64] + [_dp] * 7
        lib.ref_kepler_orbit.argtypes = [C.c_double] * 4 + [_dp] * 8
        lib.ref_direct.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double, C.c_int, C.c_int,
                                   _dp, _dp, _dp, _u64p]
        lib.ref_direct_timed.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double, C.c_int,
                                         C.c_int, C.c_int, _dp]
        lib.ref_reference_acceleration.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_size_t,
                                                   C.c_double, _dp]
        lib.ref_morton.argtypes = [C.c_size_t, _dp, _dp, _dp, C.c_int, _u64p, _u64p, _dp, _dp]
        lib.ref_spread_bits.argtypes = [C.c_uint32]
        lib.ref_spread_bits.restype = C.c_uint64
        lib.ref_morton_code_grid.argtypes = [C.c_uint32] * 3
        lib.ref_morton_code_grid.restype = C.c_uint64
        lib.ref_barnes_hut.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                       C.c_uint64, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp,
                                       _u64p, C.POINTER(C.c_void_p)]
        lib.ref_barnes_hut_timed.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double,
                                             C.c_double, C.c_uint64, C.c_int, C.c_int, C.c_int,
                                             _dp]
        lib.ref_tree_node_count.argtypes = [C.c_void_p]
        lib.ref_tree_node_count.restype = C.c_size_t
        lib.ref_tree_leaf_count.argtypes = [C.c_void_p]
        lib.ref_tree_leaf_count.restype = C.c_size_t
        lib.ref_tree_depth.argtypes = [C.c_void_p]
        lib.ref_tree_depth.restype = C.c_uint
        lib.ref_tree_copy.argtypes = [C.c_void_p, _dp, _u64p, _dp]
        lib.ref_tree_free.argtypes = [C.c_void_p]
        lib.ref_integrate_direct.argtypes = [C.c_size_t] + [_dp] * 10 + [
            C.c_double, C.c_double, C.c_uint64, C.c_int, C.c_int]
        lib.ref_potential_energy.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp, C.c_double]
        lib.ref_potential_energy.restype = C.c_double
        lib.ref_kinetic_energy.argtypes = [C.c_size_t, _dp, _dp, _dp, _dp]
        lib.ref_kinetic_energy.restype = C.c_double
        lib.ref_diagnostics.argtypes = [C.c_size_t] + [_dp] * 7 + [C.c_double, _dp]
        # Run output (ref_output_shim.cpp).
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_default_configuration.argtypes = [C.c_char_p, C.c_size_t]
        lib.ref_default_configuration.restype = C.c_size_t
        lib.ref_write_checkpoint.argtypes = [C.c_char_p, C.c_uint64, C.c_size_t] + [_dp] * 10
        lib.ref_read_checkpoint.argtypes = [C.c_char_p, _u64p, _u64p, C.c_size_t] + [_dp] * 10 + [
            C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
        lib.ref_write_trajectory.argtypes = [C.c_char_p, C.c_size_t, _dp, C.c_double, C.c_int,
                                             C.c_size_t, _u64p, _dp, _dp, _dp]
        lib.ref_read_trajectory.argtypes = [C.c_char_p, _u64p, _dp, C.POINTER(C.c_int),
                                            C.POINTER(C.c_size_t), C.c_size_t, C.c_size_t, _dp,
                                            _u64p, _dp, _dp, _dp]
        lib.ref_write_diagnostics_log.argtypes = [C.c_char_p, C.c_size_t, _u64p] + [_dp] * 5

    @staticmethod
    def available(path: str = REFERENCE_PATH) -> bool:
        return os.path.exists(path)

    # -- run output: the reference's own writers and readers ------------------

    CHECKPOINT_ARRAYS = ("m", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")

    def _raise(self, what):
        raise RuntimeError(f"{what}: {self.lib.ref_last_error().decode()}")

    def default_configuration(self) -> str:
        """sim::write_configuration of a default Configuration."""
        size = self.lib.ref_default_configuration(None, 0)
        buf = C.create_string_buffer(size + 1)
        self.lib.ref_default_configuration(buf, size)
        return buf.raw[:size].decode()

    def write_checkpoint(self, path, step, state):
        """sim::write_checkpoint of {default configuration, step, state}."""
        arrs = [np.ascontiguousarray(state[k], dtype=np.float64) for k in self.CHECKPOINT_ARRAYS]
        if self.lib.ref_write_checkpoint(os.fsencode(path), int(step), len(arrs[0]),
                                         *(_d(a) for a in arrs)) != 0:
            self._raise("write_checkpoint")

    def read_checkpoint(self, path, capacity=1 << 22):
        """sim::read_checkpoint: step, state arrays and the configuration as
        sim::write_configuration writes it back out."""
        step, n = C.c_uint64(), C.c_uint64()
        out = {k: np.zeros(capacity) for k in self.CHECKPOINT_ARRAYS}
        text = C.create_string_buffer(1 << 16)
        length = C.c_size_t()
        if self.lib.ref_read_checkpoint(os.fsencode(path), C.byref(step), C.byref(n), capacity,
                                        *(_d(out[k]) for k in self.CHECKPOINT_ARRAYS), text,
                                        1 << 16, C.byref(length)) != 0:
            self._raise("read_checkpoint")
        res = {k: v[:n.value].copy() for k, v in out.items()}
        res["step"] = step.value
        res["configuration"] = text.raw[:length.value].decode()
        return res

    def write_trajectory(self, path, masses, timestep, frames, with_velocities):
        """sim::TrajectoryWriter: `frames` is a list of (step, time, state)."""
        m = np.ascontiguousarray(masses, dtype=np.float64)
        n = len(m)
        steps = np.array([f[0] for f in frames], dtype=np.uint64)
        times = np.array([f[1] for f in frames], dtype=np.float64)
        xyz = np.concatenate([np.concatenate([f[2][k] for k in ("x", "y", "z")])
                              for f in frames]) if frames else np.zeros(1)
        v = (np.concatenate([np.concatenate([f[2][k] for k in ("vx", "vy", "vz")])
                             for f in frames]) if frames and with_velocities else np.zeros(1))
        if self.lib.ref_write_trajectory(os.fsencode(path), n, _d(m), float(timestep),
                                         int(with_velocities), len(frames), _u(steps),
                                         _d(times), _d(np.ascontiguousarray(xyz)),
                                         _d(np.ascontiguousarray(v))) != 0:
            self._raise("TrajectoryWriter")

    def write_diagnostics_log(self, path, rows):
        """sim::DiagnosticsLog: `rows` is a list of (step, time, diagnostics),
        each diagnostics a dict as `diagnostics` returns."""
        steps = np.array([r[0] for r in rows] or [0], dtype=np.uint64)
        cols = {k: np.array([r[2][k] for r in rows] or [0.0], dtype=np.float64)
                for k in ("kinetic_energy", "potential_energy")}
        vecs = {k: np.ascontiguousarray(np.concatenate([np.asarray(r[2][k], dtype=np.float64)
                                                        for r in rows]) if rows else np.zeros(3))
                for k in ("linear_momentum", "angular_momentum")}
        times = np.array([r[1] for r in rows] or [0.0], dtype=np.float64)
        if self.lib.ref_write_diagnostics_log(os.fsencode(path), len(rows), _u(steps), _d(times),
                                              _d(cols["kinetic_energy"]),
                                              _d(cols["potential_energy"]),
                                              _d(vecs["linear_momentum"]),
                                              _d(vecs["angular_momentum"])) != 0:
            self._raise("DiagnosticsLog")

    def read_trajectory(self, path, max_frames=16, max_n=4096):
        """sim::TrajectoryReader: header facts and the frames."""
        n, ts, wv, nf = C.c_uint64(), C.c_double(), C.c_int(), C.c_size_t()
        masses = np.zeros(max_n)
        steps = np.zeros(max_frames, dtype=np.uint64)
        times = np.zeros(max_frames)
        xyz = np.zeros(max_frames * 3 * max_n)
        v = np.zeros(max_frames * 3 * max_n)
        if self.lib.ref_read_trajectory(os.fsencode(path), C.byref(n), C.byref(ts), C.byref(wv),
                                        C.byref(nf), max_frames, max_n, _d(masses), _u(steps),
                                        _d(times), _d(xyz), _d(v)) != 0:
            self._raise("TrajectoryReader")
        count, frames = n.value, min(nf.value, max_frames)
        out = []
        for f in range(frames):
            p = xyz[f * 3 * count:(f + 1) * 3 * count]
            st = {"x": p[:count].copy(), "y": p[count:2 * count].copy(),
                  "z": p[2 * count:].copy()}
            if wv.value:
                q = v[f * 3 * count:(f + 1) * 3 * count]
                st.update(vx=q[:count].copy(), vy=q[count:2 * count].copy(),
                          vz=q[2 * count:].copy())
            out.append((int(steps[f]), float(times[f]), st))
        return {"n": count, "timestep": ts.value, "with_velocities": bool(wv.value),
                "masses": masses[:count].copy(), "frames": out, "frame_count": nf.value}

    def worker_count(self) -> int:
        return int(self.lib.ref_default_worker_count())

    def plummer(self, count, total_mass=1.0, scale_radius=1.0, seed=20260811):
        arrs = [np.zeros(count) for _ in range(7)]
        rc = self.lib.ref_plummer(count, total_mass, scale_radius, seed, *(_d(a) for a in arrs))
        if rc != 0:
            raise RuntimeError("reference Plummer sampler failed")
        return dict(zip(("x", "y", "z", "vx", "vy", "vz", "m"), arrs))

    def kepler_orbit(self, primary_mass=1.0, secondary_mass=1.0, semi_major_axis=1.0,
                     eccentricity=0.0):
        """initial_conditions::make_kepler_orbit and kepler_period: (state, period),
        or None where the reference refuses the parameters."""
        arrs = [np.zeros(2) for _ in range(7)]
        period = np.zeros(1)
        if self.lib.ref_kepler_orbit(primary_mass, secondary_mass, semi_major_axis, eccentricity,
                                     *(_d(a) for a in arrs), _d(period)) != 0:
            return None
        return dict(zip(("x", "y", "z", "vx", "vy", "vz", "m"), arrs)), float(period[0])

    def direct(self, x, y, z, m, softening, kernel="scalar", threads=1):
        n = len(m)
        a = [np.zeros(n) for _ in range(3)]
        pairs = np.zeros(1, np.uint64)
        self.lib.ref_direct(n, _d(x), _d(y), _d(z), _d(m), softening,
                            1 if kernel == "avx2" else 0, threads, _d(a[0]), _d(a[1]), _d(a[2]),
                            _u(pairs))
        return np.stack(a, axis=1), int(pairs[0])

    def direct_seconds(self, x, y, z, m, softening, threads, repeats=1, kernel="avx2"):
        s = C.c_double()
        self.lib.ref_direct_timed(len(m), _d(x), _d(y), _d(z), _d(m), softening,
                                  1 if kernel == "avx2" else 0, threads, repeats, C.byref(s))
        return s.value

    def reference_acceleration(self, x, y, z, m, target, softening):
        out = np.zeros(3)
        self.lib.ref_reference_acceleration(len(m), _d(x), _d(y), _d(z), _d(m), target,
                                            softening, _d(out))
        return out

    def morton(self, x, y, z, threads=1):
        n = len(x)
        codes = np.zeros(n, np.uint64)
        idx = np.zeros(n, np.uint64)
        origin = np.zeros(3)
        size = np.zeros(1)
        self.lib.ref_morton(n, _d(x), _d(y), _d(z), threads, _u(codes), _u(idx), _d(origin),
                            _d(size))
        return codes, idx, origin, float(size[0])

    def barnes_hut(self, x, y, z, m, softening, opening_angle=0.5, leaf_capacity=32,
                   quadrupole=False, kernel="scalar", threads=1, with_tree=True):
        n = len(m)
        a = [np.zeros(n) for _ in range(3)]
        counts = np.zeros(3, np.uint64)
        handle = C.c_void_p()
        self.lib.ref_barnes_hut(n, _d(x), _d(y), _d(z), _d(m), softening, opening_angle,
                                leaf_capacity, 1 if quadrupole else 0,
                                1 if kernel == "avx2" else 0, threads, _d(a[0]), _d(a[1]),
                                _d(a[2]), _u(counts), C.byref(handle) if with_tree else None)
        tree = None
        if with_tree:
            nn = self.lib.ref_tree_node_count(handle)
            reals = np.zeros((nn, 5))
            ind = np.zeros((nn, 3), np.uint64)
            quads = np.zeros((nn, 6)) if quadrupole else None
            self.lib.ref_tree_copy(handle, _d(reals), _u(ind),
                                   _d(quads) if quadrupole else None)
            tree = Tree(reals, ind, quads, self.lib.ref_tree_leaf_count(handle),
                        self.lib.ref_tree_depth(handle))
            self.lib.ref_tree_free(handle)
        return np.stack(a, axis=1), counts, tree

    def barnes_hut_seconds(self, x, y, z, m, softening, opening_angle, leaf_capacity, quadrupole,
                           threads, repeats=1):
        s = C.c_double()
        self.lib.ref_barnes_hut_timed(len(m), _d(x), _d(y), _d(z), _d(m), softening,
                                      opening_angle, leaf_capacity, 1 if quadrupole else 0,
                                      threads, repeats, C.byref(s))
        return s.value

    def integrate_direct(self, state, m, softening, dt, steps, integrator="vv", kernel="scalar"):
        s = {k: np.ascontiguousarray(v, dtype=np.float64).copy() for k, v in state.items()}
        self.lib.ref_integrate_direct(
            len(m), *(_d(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")),
            _d(m), softening, dt, steps, {"vv": 0, "yoshida4": 1, "rk4": 2}[integrator],
            1 if kernel == "avx2" else 0)
        return s

    def potential_energy(self, x, y, z, m, softening):
        return self.lib.ref_potential_energy(len(m), _d(x), _d(y), _d(z), _d(m), softening)

    def kinetic_energy(self, vx, vy, vz, m):
        return self.lib.ref_kinetic_energy(len(m), _d(vx), _d(vy), _d(vz), _d(m))

    def diagnostics(self, x, y, z, vx, vy, vz, m, softening):
        """core::measure_diagnostics: kinetic and potential energy, linear and
        angular momentum."""
        out = np.zeros(8)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, vx, vy, vz, m)]
        self.lib.ref_diagnostics(len(arrs[-1]), *(_d(a) for a in arrs), softening, _d(out))
        return {"kinetic_energy": out[0], "potential_energy": out[1],
                "linear_momentum": out[2:5].copy(), "angular_momentum": out[5:8].copy()}


class ReferenceCuda:
    """ctypes binding of ref_cuda_shim.cpp: the reference's CudaDirectSolver and
    CudaTreeSolver (its own GPU path) on this machine's device."""

    @staticmethod
    def built(single: bool = False) -> bool:
        return os.path.exists(REFERENCE_CUDA_SINGLE_PATH if single else REFERENCE_CUDA_PATH)

    def __init__(self, path: str | None = None, single: bool = False):
        """single: the reference's single-precision build (Real = float, its
        cuda-single-precision preset) instead of its double-precision one."""
        path = path or (REFERENCE_CUDA_SINGLE_PATH if single else REFERENCE_CUDA_PATH)
        lib = C.CDLL(path)
        lib.ref_cuda_real_bytes.restype = C.c_int
        self.real_bytes = lib.ref_cuda_real_bytes()
        lib.ref_cuda_direct_timed.argtypes = [C.c_size_t] + [_dp] * 4 + [
            C.c_double, C.c_int, _dp, _dp, _dp, _dp, _dp]
        lib.ref_cuda_tree_timed.argtypes = [C.c_size_t] + [_dp] * 4 + [
            C.c_double, C.c_double, C.c_uint64, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp,
            _dp, _u64p]
        self.lib = lib

    def available(self) -> bool:
        return bool(self.lib.ref_cuda_available())

    def direct_timed(self, x, y, z, m, softening, repeats=3):
        """(wall s per evaluation, kernel s per evaluation, accelerations (n, 3))."""
        x, y, z, m = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, m))
        n = len(m)
        a = [np.zeros(n) for _ in range(3)]
        wall, kern = C.c_double(), C.c_double()
        rc = self.lib.ref_cuda_direct_timed(n, _d(x), _d(y), _d(z), _d(m), softening,
                                            int(repeats), C.byref(wall), C.byref(kern),
                                            *(_d(v) for v in a))
        if rc != 0:
            raise RuntimeError("the reference's CUDA direct solver found no device")
        return wall.value, kern.value, np.stack(a, axis=1)

    def tree_timed(self, x, y, z, m, softening, opening_angle, leaf_capacity, quadrupole,
                   threads, repeats=1):
        """(wall s, kernel s, accelerations (n, 3), (pairs, cells)) per evaluation."""
        x, y, z, m = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, m))
        n = len(m)
        a = [np.zeros(n) for _ in range(3)]
        counts = np.zeros(2, np.uint64)
        wall, kern = C.c_double(), C.c_double()
        rc = self.lib.ref_cuda_tree_timed(n, _d(x), _d(y), _d(z), _d(m), softening,
                                          opening_angle, int(leaf_capacity),
                                          1 if quadrupole else 0, int(threads), int(repeats),
                                          C.byref(wall), C.byref(kern), *(_d(v) for v in a),
                                          _u(counts))
        if rc != 0:
            raise RuntimeError("the reference's CUDA tree solver found no device")
        return wall.value, kern.value, np.stack(a, axis=1), (int(counts[0]), int(counts[1]))


REFERENCE_ADAPTER_PATH = os.path.join(HERE, "_ref", "libref_adapter.so")


class AdapterDriver:
    """ctypes binding of ref_adapter_shim.cpp: the reference's own integrators
    (VelocityVerlet, Yoshida4, RungeKutta4) driven over the reference's CPU
    solvers or over the B200 ForceSolver adapters, or B200Integrator."""

    FIELDS = {"reference-direct": 0, "reference-tree": 1, "b200-direct": 2, "b200-tree": 3}
    METHODS = {"vv": 0, "yoshida4": 1, "rk4": 2}
    PRECISIONS = {"fp32": 0, "split": 1, "fp64": 2}
    STATE = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")

    @staticmethod
    def built() -> bool:
        return os.path.exists(REFERENCE_ADAPTER_PATH)

    def __init__(self, path: str = REFERENCE_ADAPTER_PATH):
        lib = C.CDLL(path)
        lib.ra_last_error.restype = C.c_char_p
        lib.ra_try_create.argtypes = [C.c_int, C.c_int]
        lib.ra_integrator_traits.argtypes = [C.c_int, C.c_int, C.c_char_p, C.c_size_t,
                                             C.POINTER(C.c_int), C.POINTER(C.c_int), _u64p]
        lib.ra_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                               C.c_uint64, C.c_int, C.c_size_t] + [_dp] * 10 + [
            C.c_double, C.c_uint64, _u64p, C.c_char_p, C.c_size_t]
        self.lib = lib

    def last_error(self) -> str:
        return self.lib.ra_last_error().decode()

    def try_create(self, tree: bool, precision: str = "fp32") -> int:
        """1: a solver; 0: null (no usable device); other: an error code."""
        return self.lib.ra_try_create(int(tree), self.PRECISIONS[precision])

    def traits(self, adapter: bool, method: str):
        name = C.create_string_buffer(64)
        order, symplectic = C.c_int(), C.c_int()
        evaluations = np.zeros(1, np.uint64)
        self.lib.ra_integrator_traits(int(adapter), self.METHODS[method], name, 64,
                                      C.byref(order), C.byref(symplectic), _u(evaluations))
        return name.value.decode(), order.value, bool(symplectic.value), int(evaluations[0])

    def run(self, field, state, m, dt, steps, method="vv", precision="fp64",
            device_integrator=False, softening=0.01, opening_angle=0.5, leaf_capacity=32,
            quadrupole=False):
        """(return code, final state dict, counts (evaluations, pairs, cells), field name).

        The accelerations are established by the field before the first step
        (integrators::refresh_accelerations); any given in `state` are ignored."""
        n = len(m)
        arrays = {k: np.ascontiguousarray(state[k], dtype=np.float64).copy()
                  for k in ("x", "y", "z", "vx", "vy", "vz")}
        for k in ("ax", "ay", "az"):
            arrays[k] = np.zeros(n)
        mass = np.ascontiguousarray(m, dtype=np.float64)
        counts = np.zeros(3, np.uint64)
        name = C.create_string_buffer(64)
        rc = self.lib.ra_run(self.FIELDS[field], self.PRECISIONS[precision], self.METHODS[method],
                             int(device_integrator), softening, opening_angle, leaf_capacity,
                             int(quadrupole), n, *(_d(arrays[k]) for k in self.STATE), _d(mass),
                             dt, steps, _u(counts), name, 64)
        return rc, arrays, tuple(int(c) for c in counts), name.value.decode()
