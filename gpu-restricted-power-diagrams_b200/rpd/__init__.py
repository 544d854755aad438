"""Python host side of the B200 restricted power diagram engine.

A thin ctypes layer over ``librpd.so`` (declared in ``include/rpd.h``) that
mirrors the reference's host interface for the hot path: ``KNearests``
(knearests.h:9-50), ``Grid`` (Grid.h:14-70) and ``VoroAlgo``
(voronoi.h:105-256), with the same member names, argument meaning and
bool-return error behaviour.  Device work always runs in the CUDA library;
there is no CPU fallback: constructing a context without the library or
without an sm_100 device raises.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import weakref

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "librpd.so")

RPD_OK = 0
RPD_HOST, RPD_DEVICE = 0, 1
NO_CELL_LIMITS = -100000.0
STATUS_NAMES = [
    "vertex_overflow", "plane_overflow", "inconsistent_boundary", "security_radius_not_reached",
    "success", "needs_exact_predicates", "empty_cell", "find_another_beginning_vertex",
    "triangle_overflow", "seed_on_border", "hessian_overflow",
]
SUCCESS = 4
ERROR_NAMES = {0: "ok", -1: "invalid", -2: "cuda", -3: "no_device", -4: "oom", -5: "io", -6: "format",
               -7: "degenerate", -8: "capacity"}


class RpdError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"rpd error {code} ({ERROR_NAMES.get(code, '?')}): {msg}")
        self.code = code


_lib = None

# Live library objects, closed in dependency order when the interpreter exits
# (servers, batches and solvers before the contexts and grids they use), so
# that no handle is released after the library or the CUDA runtime is torn
# down.
_live = {kind: weakref.WeakSet() for kind in ("server", "batch", "solver", "grid", "context")}


def _track(kind, obj):
    _live[kind].add(obj)


@atexit.register
def _close_all():
    for kind in ("server", "batch", "solver", "grid", "context"):
        for obj in list(_live[kind]):
            try:
                obj.close()
            except Exception:
                pass

# rpd_part_reduce_fn: (sums, nsum, maxes, nmax, user) -> 0
PART_REDUCE = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_longlong), C.c_int, C.POINTER(C.c_longlong), C.c_int, C.c_void_p)


def part_range(n: int, part: int, parts: int):
    """rpd_solver_part_range: (first, count) of part `part` of `parts` of an
    n-seed diagram's stored seeds."""
    a, b = C.c_int(0), C.c_int(0)
    rc = lib().rpd_solver_part_range(n, part, parts, C.byref(a), C.byref(b))
    if rc != 0:
        raise RpdError(rc, "part range")
    return a.value, b.value


def lib():
    """Loads librpd.so (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RpdError(-2, f"{LIB_PATH} missing: build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        L.rpd_context_create.restype = C.c_void_p
        L.rpd_context_create.argtypes = [C.c_int, C.POINTER(C.c_int)]
        L.rpd_context_destroy.argtypes = [C.c_void_p]
        L.rpd_context_error.restype = C.c_char_p
        L.rpd_context_error.argtypes = [C.c_void_p]
        L.rpd_context_stream.restype = C.c_void_p
        L.rpd_context_stream.argtypes = [C.c_void_p]
        L.rpd_version.restype = C.c_char_p
        L.rpd_context_knn_variant.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.rpd_solver_create.restype = C.c_void_p
        L.rpd_solver_create.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.rpd_solver_destroy.argtypes = [C.c_void_p]
        for name in ("rpd_solver_num_points", "rpd_solver_bin_dim"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.rpd_solver_set_points.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.rpd_server_create.restype = C.c_void_p
        L.rpd_server_create.argtypes = [C.c_int, C.c_int, C.c_size_t, C.POINTER(C.c_int)]
        L.rpd_server_destroy.argtypes = [C.c_void_p]
        L.rpd_server_submit_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.POINTER(C.c_int)]
        L.rpd_server_submit_reweight.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.rpd_server_submit_solve_hessian.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                                      C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        L.rpd_server_submit_reweight_hessian.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                         C.c_void_p, C.c_void_p]
        L.rpd_server_submit_solve_blob.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.POINTER(C.c_int)]
        L.rpd_server_submit_solve_field.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.POINTER(C.c_int)]
        L.rpd_server_wait.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.rpd_server_release.argtypes = [C.c_void_p, C.c_int]
        L.rpd_server_bytes_in_use.restype = C.c_size_t
        L.rpd_server_bytes_in_use.argtypes = [C.c_void_p]
        L.rpd_solver_set_weights.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_solver_used_count.argtypes = [C.c_void_p]
        L.rpd_solver_get_used.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_solver_get_permutation.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_solver_knn.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_float)]
        L.rpd_grid_create.restype = C.c_void_p
        L.rpd_grid_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                      C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
        L.rpd_grid_load.restype = C.c_void_p
        L.rpd_grid_load.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
        L.rpd_grid_save.argtypes = [C.c_void_p, C.c_char_p]
        L.rpd_grid_valid.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.rpd_grid_volume.restype = C.c_double
        L.rpd_grid_volume.argtypes = [C.c_void_p]
        L.rpd_grid_invariants.argtypes = [C.c_void_p, C.c_void_p]
        L.rpd_grid_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4
        L.rpd_grid_export.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.rpd_grid_destroy.argtypes = [C.c_void_p]
        L.rpd_grid_make_blob.restype = C.c_void_p
        L.rpd_grid_make_blob.argtypes = [C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_int)]
        L.rpd_grid_make_cube.restype = C.c_void_p
        L.rpd_grid_make_cube.argtypes = [C.c_int, C.POINTER(C.c_int)]
        L.rpd_params_default.argtypes = [C.c_void_p]
        L.rpd_solver_set_grid.argtypes = [C.c_void_p, C.c_void_p]
        L.rpd_solver_launch.argtypes = [C.c_void_p, C.c_void_p]
        L.rpd_solver_get_moments.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_solver_get_status.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_solver_get_stats.argtypes = [C.c_void_p, C.c_void_p]
        L.rpd_solver_trace_cell.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_solver_get_hessian.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_compare_moments.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
        L.rpd_solver_set_grid_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.rpd_solver_set_grid_blob.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64]
        L.rpd_solver_export_grid.restype = C.c_void_p
        L.rpd_solver_export_grid.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.rpd_batch_create.restype = C.c_void_p
        L.rpd_batch_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.rpd_batch_launch.argtypes = [C.c_void_p]
        L.rpd_batch_get_stats.argtypes = [C.c_void_p, C.c_void_p]
        L.rpd_batch_destroy.argtypes = [C.c_void_p]
        L.rpd_solver_part_range.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.rpd_solver_launch_part.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, PART_REDUCE, C.c_void_p]
        L.rpd_solver_get_stored.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.rpd_solver_set_stored.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_seeds_load.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_float)),
                                     C.POINTER(C.c_int)]
        L.rpd_seeds_free.argtypes = [C.POINTER(C.c_float)]
        L.rpd_seeds_save_binary.argtypes = [C.c_char_p, C.c_void_p, C.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


FLAG_FIRST_PASS_ONLY = 1
FLAG_COUNTERS = 2
FLAG_NO_EARLY_OUT = 4
FLAG_NO_DEFER = 8
FLAG_REFERENCE_APEX = 16
FLAG_FRESH_NEIGHBOURS = 32
FLAG_NO_PROBE = 64
FLAG_NO_T_AHEAD = 128
FLAG_KNN_WARP = 256
FLAG_SAFE_RADIUS = 1024
FLAG_OUTSIDE_PROBE = 2048
FLAG_KNN_THREAD = 512
PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_FP32 = 2
COUNTER_NAMES = ["planes_tested", "clips", "vertex_tests", "vertices_made", "boundary_cells", "triangles",
                 "exports", "export_vertices", "outside_early", "cone_empty", "cones_skipped",
                 "escalated_tests", "escalated_vertices", "escalated_radii", "start_corner_cells"]


class Params(C.Structure):
    """rpd_params: the VoroAlgo knobs (voronoi.h:199-246)."""

    _fields_ = [("K", C.c_int), ("P", C.c_int), ("V", C.c_int), ("T", C.c_int), ("max_extra_passes", C.c_int),
                ("cube_eps", C.c_float), ("out_domain", C.c_int), ("flags", C.c_uint),
                ("keep_distance", C.c_int), ("keep_volume", C.c_double), ("hessian_h", C.c_int),
                ("hessian_hc", C.c_int), ("precision", C.c_int)]

    @classmethod
    def default(cls, **kw):
        p = cls()
        lib().rpd_params_default(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        return p


class Stats(C.Structure):
    _fields_ = [("npasses", C.c_int), ("pass_cells", C.c_int * 8), ("pass_K", C.c_int * 8),
                ("pass_P", C.c_int * 8), ("pass_V", C.c_int * 8), ("pass_T", C.c_int * 8),
                ("pass_knn_ms", C.c_float * 8), ("pass_cell_ms", C.c_float * 8), ("status_hist", C.c_int * 11),
                ("counters", C.c_ulonglong * 15), ("knn_candidates", C.c_ulonglong), ("total_ms", C.c_float),
                ("kernel_launches", C.c_int), ("pass_cell_kernel_ms", C.c_float * 8), ("probe_outside", C.c_int),
                ("probe_ms", C.c_float), ("pass_knn_variant", C.c_int * 8)]

    def as_dict(self):
        n = self.npasses
        return {
            "npasses": n,
            "passes": [{"cells": self.pass_cells[i], "K": self.pass_K[i], "P": self.pass_P[i], "V": self.pass_V[i],
                        "T": self.pass_T[i], "knn_ms": self.pass_knn_ms[i], "cell_ms": self.pass_cell_ms[i],
                        "cell_kernel_ms": self.pass_cell_kernel_ms[i],
                        "knn_variant": ("warp", "thread")[self.pass_knn_variant[i]]}
                       for i in range(min(n, 8))],
            "status": {STATUS_NAMES[i]: v for i, v in enumerate(self.status_hist) if v},
            "counters": {COUNTER_NAMES[i]: int(v) for i, v in enumerate(self.counters)},
            "knn_candidates": int(self.knn_candidates),
            "total_ms": self.total_ms,
            "kernel_launches": self.kernel_launches,
            "probe_outside": self.probe_outside,
            "probe_ms": self.probe_ms,
        }


class Context:
    """A CUDA device bound to the engine (OpenCLContext in the reference)."""

    def __init__(self, device: int = 0):
        err = C.c_int(0)
        self.h = lib().rpd_context_create(device, C.byref(err))
        if not self.h:
            raise RpdError(err.value, f"no usable sm_100 device {device}")
        _track("context", self)

    def error(self) -> str:
        return lib().rpd_context_error(self.h).decode()

    def knn_variant(self, K: int, variant: int = -2) -> int:
        """rpd_context_knn_variant: pin (0 warp, 1 thread per seed), forget
        (-1) or read (-2) the neighbour-search variant for K."""
        rc = lib().rpd_context_knn_variant(self.h, K, variant)
        if rc < -1:
            self.check(rc)
        return rc

    def check(self, rc):
        if rc != RPD_OK:
            raise RpdError(rc, self.error())

    def close(self):
        if self.h:
            lib().rpd_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def load_seeds(path, points4d: bool = False, binary: bool = False) -> np.ndarray:
    """A seed file through the library's loader (rpd_seeds_load): the
    reference's text .xyz format (Utils::loadSeedsFile, Utils.cpp:36-79; a
    weight column with points4d) or its binary format (binary=True,
    readBinarySeedsFile, Utils.cpp:81-97).  Returns (n, 4) float32 x y z w
    in the reference frame, not normalised."""
    p = C.POINTER(C.c_float)()
    n = C.c_int(0)
    rc = lib().rpd_seeds_load(os.fsencode(str(path)), int(points4d), int(binary), C.byref(p), C.byref(n))
    if rc != 0:
        raise RpdError(rc, f"could not load seeds from {path}")
    try:
        return np.ctypeslib.as_array(p, shape=(n.value, 4)).copy()
    finally:
        lib().rpd_seeds_free(p)


def save_seeds_binary(path, xyzw) -> None:
    """saveBinarySeedsFile (Utils.cpp:99-113) through rpd_seeds_save_binary."""
    x = as_xyzw(xyzw)
    rc = lib().rpd_seeds_save_binary(os.fsencode(str(path)), _ptr(x), len(x))
    if rc != 0:
        raise RpdError(rc, f"could not save seeds to {path}")


def as_xyzw(points) -> np.ndarray:
    a = np.asarray(points, dtype=np.float32)
    if a.ndim == 1:
        a = a.reshape(-1, 4)
    if a.shape[1] == 3:
        a = np.concatenate([a, np.zeros((len(a), 1), np.float32)], axis=1)
    return np.ascontiguousarray(a, dtype=np.float32)


class Solver:
    """A resident seed set on the device (the state VoroAlgo keeps between
    setInputPoints and launch)."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        err = C.c_int(0)
        self.h = lib().rpd_solver_create(self.ctx.h, C.byref(err))
        if not self.h:
            raise RpdError(err.value, self.ctx.error())
        _track("solver", self)

    def set_points(self, xyzw):
        x = as_xyzw(xyzw)
        self.ctx.check(lib().rpd_solver_set_points(self.h, _ptr(x), len(x), RPD_HOST))
        return self

    def used(self):
        """Used cells of the last launch with keep_distance >= 0 and a grid:
        (rows (m,4) in ascending user order, user ids (m,)), the reference's
        compressed output (getBarycenters + getPermutationToUser)."""
        m = lib().rpd_solver_used_count(self.h)
        if m < 0:
            raise RpdError(m, "no used cells: launch with keep_distance >= 0 and a grid")
        rows = np.zeros((max(m, 1), 4), np.float64)
        ids = np.zeros(max(m, 1), np.int32)
        rc = lib().rpd_solver_get_used(self.h, _ptr(rows), _ptr(ids), RPD_HOST)
        if rc < 0:
            self.ctx.check(rc)
        return rows[:m], ids[:m]

    def set_weights(self, w):
        """Weight-only re-solve setup: new weights (user order) for the seeds
        already set; bins and the last neighbour table (same K) are kept."""
        w = np.ascontiguousarray(w, np.float32)
        if w.shape != (self.n,):
            raise ValueError(f"expected {self.n} weights, got shape {w.shape}")
        self.ctx.check(lib().rpd_solver_set_weights(self.h, _ptr(w), RPD_HOST))
        return self

    @property
    def n(self) -> int:
        return lib().rpd_solver_num_points(self.h)

    @property
    def dim(self) -> int:
        return lib().rpd_solver_bin_dim(self.h)

    def permutation(self) -> np.ndarray:
        out = np.zeros(self.n, np.int32)
        self.ctx.check(lib().rpd_solver_get_permutation(self.h, _ptr(out), RPD_HOST))
        return out

    def set_grid(self, grid):
        self.ctx.check(lib().rpd_solver_set_grid(self.h, grid.h if grid is not None else None))
        self._grid = grid
        return self

    def set_grid_blob(self, size, nellipsoids=5, seed=2):
        """The seeded blob of Grid.blob, built on the device."""
        self.ctx.check(lib().rpd_solver_set_grid_blob(self.h, int(size), int(nellipsoids), int(seed)))
        self._grid = None
        return self

    def set_grid_field(self, field):
        """The domain {field < 0} of a field on the (S+1)^3 corner lattice
        (numpy (S+1, S+1, S+1) indexed [z, y, x], or flat x-fastest), built
        on the device."""
        f = np.ascontiguousarray(field, np.float32).reshape(-1)
        s1 = round(len(f) ** (1.0 / 3.0))
        if s1 ** 3 != len(f) or s1 < 2:
            raise ValueError("field must hold (S+1)^3 values")
        self.ctx.check(lib().rpd_solver_set_grid_field(self.h, s1 - 1, _ptr(f), RPD_HOST))
        self._grid = None
        return self

    def export_grid(self):
        """The solver's domain as a host Grid."""
        err = C.c_int(0)
        h = lib().rpd_solver_export_grid(self.h, C.byref(err))
        if not h:
            raise RpdError(err.value, self.ctx.error())
        return Grid(h)

    def launch(self, params=None, **kw):
        p = params if params is not None else Params.default(**kw)
        self.ctx.check(lib().rpd_solver_launch(self.h, C.byref(p)))
        return self

    def launch_part(self, part: int, parts: int, reduce, params=None, **kw):
        """rpd_solver_launch_part: the cells of this part's stored range, with
        the retry schedule of the whole diagram.  reduce(sums, maxes) gets this
        part's counts (int64 arrays) and returns them summed (maximised) over
        every part."""
        p = params if params is not None else Params.default(**kw)
        err = []

        def cb(sums, nsum, maxes, nmax, user):
            try:
                s = np.ctypeslib.as_array(sums, shape=(nsum,))
                m = np.ctypeslib.as_array(maxes, shape=(nmax,))
                rs, rm = reduce(s.copy(), m.copy())
                s[:] = rs
                m[:] = rm
                return 0
            except Exception as exc:  # reported after the launch returns
                err.append(exc)
                return 1

        fn = PART_REDUCE(cb)
        rc = lib().rpd_solver_launch_part(self.h, C.byref(p), part, parts, fn, None)
        if err:
            raise err[0]
        self.ctx.check(rc)
        return self

    def stored(self, first: int, count: int, out=None, status=None, device: bool = False):
        """rpd_solver_get_stored: results of stored seeds first .. first+count-1
        ((count, 4) doubles, (count,) statuses); with device=True, out and
        status are device pointers (ints) filled in place."""
        if device:
            self.ctx.check(lib().rpd_solver_get_stored(self.h, C.c_void_p(out), C.c_void_p(status), first, count,
                                                      RPD_DEVICE))
            return None
        o = np.zeros((count, 4), np.float64)
        st = np.zeros(count, np.int32)
        self.ctx.check(lib().rpd_solver_get_stored(self.h, _ptr(o), _ptr(st), first, count, RPD_HOST))
        return o, st

    def set_stored(self, out, status, device: bool = False):
        """rpd_solver_set_stored: installs every stored seed's results."""
        if device:
            self.ctx.check(lib().rpd_solver_set_stored(self.h, C.c_void_p(out), C.c_void_p(status), RPD_DEVICE))
        else:
            o = np.ascontiguousarray(out, np.float64)
            st = np.ascontiguousarray(status, np.int32)
            self.ctx.check(lib().rpd_solver_set_stored(self.h, _ptr(o), _ptr(st), RPD_HOST))
        return self

    def moments(self) -> np.ndarray:
        out = np.zeros((self.n, 4), np.float64)
        self.ctx.check(lib().rpd_solver_get_moments(self.h, _ptr(out), RPD_HOST))
        return out

    def status(self) -> np.ndarray:
        out = np.zeros(self.n, np.int32)
        self.ctx.check(lib().rpd_solver_get_status(self.h, _ptr(out), RPD_HOST))
        return out

    def stats(self) -> dict:
        st = Stats()
        self.ctx.check(lib().rpd_solver_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def hessian(self, H: int, HC: int = 1):
        """Hessian rows of the last launch with hessian_h=H, hessian_hc=HC:
        (values (n,H) areas for HC=1 or (n,H,4) area-weighted centroids and
        areas, ids (n,H) neighbour user ids, -1 after a row's last facet).
        With used cells: the used cells' rows, ids their compacted positions."""
        m = lib().rpd_solver_used_count(self.h)
        rows = m if m >= 0 else self.n
        vals = np.zeros((max(rows, 1), H, HC), np.float64)
        ids = np.zeros((max(rows, 1), H), np.int32)
        self.ctx.check(lib().rpd_solver_get_hessian(self.h, _ptr(vals), _ptr(ids), RPD_HOST))
        vals, ids = vals[:rows], ids[:rows]
        return (vals[:, :, 0] if HC == 1 else vals), ids

    TRACE_KINDS = {0: "seed", 1: "plane", 2: "cavity", 3: "vertex", 4: "integrate", 5: "start", 6: "triangle"}

    def trace_cell(self, user_id: int, params=None, cap: int = 20000, **kw):
        """Debugging: the clip/integration records of one seed's cell."""
        p = params if params is not None else Params.default(**kw)
        rec = np.zeros((cap, 12), np.float64)
        n = lib().rpd_solver_trace_cell(self.h, int(user_id), C.byref(p), _ptr(rec), cap)
        if n < 0:
            raise RpdError(n, self.ctx.error())
        return rec[:n]

    def knn(self, K: int, return_ms: bool = False):
        out = np.zeros((self.n, K), np.int32)
        ms = C.c_float(0)
        self.ctx.check(lib().rpd_solver_knn(self.h, K, _ptr(out), RPD_HOST, C.byref(ms)))
        return (out, ms.value) if return_ms else out

    def close(self):
        if self.h:
            lib().rpd_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MomentDiff(C.Structure):
    _fields_ = [("cells", C.c_longlong), ("cells_both", C.c_longlong), ("sum_a", C.c_double * 4),
                ("sum_b", C.c_double * 4), ("max_mass", C.c_double), ("max_bary", C.c_double * 3),
                ("max_moment", C.c_double * 3), ("avg_mass", C.c_double), ("avg_bary", C.c_double * 3),
                ("avg_moment", C.c_double * 3)]


def compare_moments(a, b) -> dict:
    """rpd_compare_moments: the reference diff tool's figures for two (n,4)
    moment arrays (m*x, m*y, m*z, m)."""
    a = np.ascontiguousarray(a, np.float64).reshape(-1, 4)
    b = np.ascontiguousarray(b, np.float64).reshape(-1, 4)
    if a.shape != b.shape:
        raise ValueError("moment arrays differ in size")
    d = MomentDiff()
    rc = lib().rpd_compare_moments(_ptr(a), _ptr(b), len(a), C.byref(d))
    if rc != RPD_OK:
        raise RpdError(rc, "compare_moments")
    out = {}
    for k, _ in d._fields_:
        v = getattr(d, k)
        out[k] = list(v) if hasattr(v, "__len__") else v
    return out


class BatchStats(C.Structure):
    _fields_ = [("diagrams", C.c_int), ("cells", C.c_longlong), ("graph_ms", C.c_float),
                ("passes_captured", C.c_int), ("max_passes", C.c_int), ("kernel_launches", C.c_int),
                ("captures", C.c_int), ("solved_alone", C.c_int), ("pass0_knn_ms", C.c_float),
                ("pass0_cell_kernel_ms", C.c_float), ("pass_ms", C.c_float * 8), ("pass_cells", C.c_longlong * 8),
                ("probe_ms", C.c_float), ("probe_outside", C.c_longlong), ("knn_variant", C.c_int * 6),
                ("knn_trial_warp_ms", C.c_float * 6), ("knn_trial_thread_ms", C.c_float * 6)]

    def as_dict(self):
        arrays = ("pass_ms", "pass_cells", "knn_variant", "knn_trial_warp_ms", "knn_trial_thread_ms")
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in arrays}
        n = min(self.passes_captured, 8)
        d["passes"] = [{"cells": int(self.pass_cells[i]), "ms": self.pass_ms[i]} for i in range(n)]
        d["knn_classes"] = [{"K_max": 32 * s, "variant": ("warp", "thread")[v] if v >= 0 else None,
                             "trial_warp_ms": self.knn_trial_warp_ms[c], "trial_thread_ms": self.knn_trial_thread_ms[c]}
                            for c, (s, v) in enumerate(zip((1, 2, 3, 4, 6, 8), self.knn_variant)) if v >= 0]
        return d


class Batch:
    """Many independent diagrams solved together (rpd_batch_*): every pass of
    every solver in shared launches, the whole solve one CUDA graph replayed
    at each launch.  Each solver afterwards holds the results its own
    launch(params) would give."""

    def __init__(self, solvers, params=None, ctx: Context | None = None):
        self.solvers = list(solvers)
        self.ctx = ctx or self.solvers[0].ctx
        n = len(self.solvers)
        hs = (C.c_void_p * n)(*[s.h for s in self.solvers])
        if params is None:
            pa = None
        else:
            if isinstance(params, Params):
                params = [params] * n
            pa = (Params * n)(*params)
        err = C.c_int(0)
        self.h = lib().rpd_batch_create(self.ctx.h, hs, pa, n, C.byref(err))
        if not self.h:
            raise RpdError(err.value, self.ctx.error())
        self._keep = (hs, pa)
        _track("batch", self)

    def launch(self):
        self.ctx.check(lib().rpd_batch_launch(self.h))
        return self

    def stats(self) -> dict:
        st = BatchStats()
        self.ctx.check(lib().rpd_batch_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def close(self):
        if self.h:
            lib().rpd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KNearests:
    """Mirror of the reference KNearests (knearests.h:9-50): the constructor
    bins the points; buildKnearests(K) computes every seed's K nearest."""

    def __init__(self, points, ctx: Context | None = None):
        self._s = Solver(ctx).set_points(points)
        self._nearest = None

    def getNumPoints(self) -> int:
        return self._s.n

    def getPermutation(self) -> np.ndarray:
        return self._s.permutation()

    def buildKnearests(self, K: int) -> bool:
        self._nearest = self._s.knn(K)
        return True

    def getNearests(self) -> np.ndarray:
        """K nearest other seeds of every seed, in user ids (user order)."""
        return self._nearest


class Grid:
    """Mirror of the reference Grid (Grid.h:14-70): a volume domain in the
    --grid layout, held by librpd (host memory)."""

    def __init__(self, handle=None):
        self.h = handle
        _track("grid", self)

    @classmethod
    def from_arrays(cls, size, in_domain, points, triangles, tri_list, offsets):
        d = np.ascontiguousarray(in_domain, dtype=np.int8)
        p = np.ascontiguousarray(np.asarray(points, np.float32)[:, :3])
        t = np.ascontiguousarray(triangles, dtype=np.int32).reshape(-1)
        tl = np.ascontiguousarray(tri_list, dtype=np.int32)
        o = np.ascontiguousarray(offsets, dtype=np.int32)
        err = C.c_int(0)
        h = lib().rpd_grid_create(int(size), _ptr(d), _ptr(p), len(p), _ptr(t), len(t) // 3, _ptr(tl), len(tl),
                                  _ptr(o), C.byref(err))
        if not h:
            raise RpdError(err.value, "bad grid arrays")
        return cls(h)

    @classmethod
    def blob(cls, size, nellipsoids=5, seed=2):
        err = C.c_int(0)
        h = lib().rpd_grid_make_blob(size, nellipsoids, seed, C.byref(err))
        if not h:
            raise RpdError(err.value, "blob")
        return cls(h)

    @classmethod
    def cube(cls, size):
        err = C.c_int(0)
        h = lib().rpd_grid_make_cube(size, C.byref(err))
        if not h:
            raise RpdError(err.value, "cube")
        return cls(h)

    def load(self, path) -> bool:
        """Grid::load (Grid.cpp:186-278); False when the file is unreadable."""
        err = C.c_int(0)
        h = lib().rpd_grid_load(str(path).encode(), C.byref(err))
        if not h:
            return False
        self.close()
        self.h = h
        return True

    def save(self, path) -> bool:
        return lib().rpd_grid_save(self.h, str(path).encode()) == RPD_OK

    def valid(self, return_reason=False):
        buf = C.create_string_buffer(256)
        ok = lib().rpd_grid_valid(self.h, buf, 256) == 1
        return (ok, buf.value.decode()) if return_reason else ok

    def getVolume(self) -> float:
        return lib().rpd_grid_volume(self.h)

    def invariants(self) -> np.ndarray:
        out = np.zeros(4, np.float64)
        lib().rpd_grid_invariants(self.h, _ptr(out))
        return out

    def info(self):
        v = [C.c_int(0) for _ in range(4)]
        lib().rpd_grid_info(self.h, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    def arrays(self):
        size, npts, ntri, nlist = self.info()
        d = np.zeros(size ** 3, np.int8)
        p = np.zeros((npts, 3), np.float32)
        t = np.zeros((ntri, 3), np.int32)
        tl = np.zeros(nlist, np.int32)
        o = np.zeros(size ** 3 + 1, np.int32)
        lib().rpd_grid_export(self.h, _ptr(d), _ptr(p), _ptr(t), _ptr(tl), _ptr(o))
        return {"size": size, "in_domain": d, "points": p, "triangles": t, "tri_list": tl, "offsets": o}

    def close(self):
        if self.h:
            lib().rpd_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VoroAlgoStat(dict):
    """One pass record (VoroAlgoStat, voronoi.h:60-103)."""


class VoroAlgo:
    """Mirror of the reference VoroAlgo (voronoi.h:105-256).

    Set the public knobs, call setInputPoints (and setGrid), then
    launch(saveData, stats): saveData(algo) reads the getters and returns a
    bool, as in the reference; results stay available afterwards too.
    """

    def __init__(self, ctx: Context | None = None, debug: bool = False):
        self.m_K, self.m_P, self.m_T, self.m_V = 25, 35, 100, 40  # voronoi.cpp:1042-1045
        self.m_maxKComputed = 100000
        self.m_vhsAlgo = [1, 2]
        self.m_keepDistance = 1
        self.m_keepVolume = 1.0
        self.m_PGlobalPercent = 0.0
        self.m_H, self.m_HC = 0, 1
        self.max_extra_passes = 5
        self.debug = debug
        self._s = Solver(ctx)
        self._grid = None
        self._n = 0

    def setInputPoints(self, seeds):
        self._s.set_points(seeds)
        self._n = self._s.n

    def setGrid(self, grid: Grid):
        self._grid = grid
        self._s.set_grid(grid)

    def getNumInputPoints(self) -> int:
        return self._n

    def launch(self, saveData=None, stats=None) -> bool:
        try:
            self._s.launch(Params.default(K=self.m_K, P=self.m_P, V=self.m_V, T=self.m_T,
                                          max_extra_passes=self.max_extra_passes))
        except RpdError:
            return False
        if stats is not None:
            d = self._s.stats()
            names = ["first"] + ["extra"] * (d["npasses"] - 1)
            for name, ps in zip(names, d["passes"]):
                stats.append(VoroAlgoStat(name=name, knn=ps["knn_ms"] / 1e3, CC=ps["cell_ms"] / 1e3,
                                          time=(ps["knn_ms"] + ps["cell_ms"]) / 1e3, nbcells=ps["cells"]))
        if saveData is not None:
            return bool(saveData(self))
        return True

    def getNumOutputPoints(self) -> int:
        return self._n

    def getBarycenters(self) -> np.ndarray:
        """(n,4) float64 (m*x, m*y, m*z, m), in user order (so
        getPermutationToUser is the identity)."""
        return self._s.moments()

    def getPermutationToUser(self) -> np.ndarray:
        return np.arange(self._n, dtype=np.int32)

    def getStatus(self) -> np.ndarray:
        return self._s.status()

    def getStats(self) -> dict:
        return self._s.stats()


class RequestInfo(C.Structure):
    """rpd_request_info: outcome and timings of one served request."""
    _fields_ = [("status", C.c_int), ("session", C.c_int), ("n", C.c_int), ("slot", C.c_int),
                ("queue_ms", C.c_double), ("latency_ms", C.c_double), ("device_ms", C.c_double),
                ("npasses", C.c_int), ("admitted_at_ms", C.c_double), ("done_at_ms", C.c_double),
                ("failed_cells", C.c_int), ("error", C.c_char * 160), ("status_hist", C.c_int * 11),
                ("last_caps", C.c_int * 4)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["error"] = self.error.decode(errors="replace")
        d["status_hist"] = {STATUS_NAMES[i]: v for i, v in enumerate(self.status_hist) if v}
        d["last_caps"] = dict(zip("KPVT", list(self.last_caps)))
        return d


class Server:
    """The serving loop of include/rpd.h (rpd_server_*): sessions kept on the
    device, solved and re-solved (weights only) on `slots` concurrent streams,
    admitted in arrival order within `mem_budget` bytes (0: 90% of the free
    device memory).  solve()/reweight() return a ticket at once; wait(ticket)
    returns (moments in user order, request info)."""

    def __init__(self, device: int = 0, slots: int = 4, mem_budget: int = 0):
        err = C.c_int(0)
        self.h = lib().rpd_server_create(device, slots, mem_budget, C.byref(err))
        if not self.h:
            raise RpdError(err.value, "server create")
        _track("server", self)
        self._out = {}     # ticket -> moments buffer (kept alive until waited for)
        self._grids = []   # grids used: they must outlive the server

    @staticmethod
    def _hessian_buffers(n, p):
        if p.hessian_h <= 0:
            return None
        return (np.zeros((n, p.hessian_h, p.hessian_hc), np.float64), np.zeros((n, p.hessian_h), np.int32))

    def solve(self, xyzw, grid=None, params=None, blob=None, field=None, **kw):
        """Submits a new session's solve; returns (ticket, session).  The
        domain: a host Grid (shared by the sessions on it), or one built on
        the device for this session alone -- blob=(size, nellipsoids, seed)
        (rpd_grid_make_blob's domain) or field= an (S+1)^3 corner-lattice
        field, domain {field < 0} (Solver.set_grid_field's layout).  With
        hessian_h > 0 the request also returns its Hessian rows (wait)."""
        if sum(d is not None for d in (grid, blob, field)) > 1:
            raise ValueError("one domain: grid, blob or field")
        x = as_xyzw(xyzw)
        p = params if params is not None else Params.default(**kw)
        out = np.zeros((len(x), 4), np.float64)
        hb = self._hessian_buffers(len(x), p)
        hv, hi = (_ptr(hb[0]), _ptr(hb[1])) if hb else (None, None)
        sess = C.c_int(-1)
        if blob is not None:
            size, nell, seed = blob
            t = lib().rpd_server_submit_solve_blob(self.h, _ptr(x), len(x), int(size), int(nell), int(seed),
                                                   C.byref(p), _ptr(out), hv, hi, C.byref(sess))
        elif field is not None:
            f = np.ascontiguousarray(field, np.float32).reshape(-1)
            s1 = round(len(f) ** (1.0 / 3.0))
            if s1 ** 3 != len(f) or s1 < 2:
                raise ValueError("field must hold (S+1)^3 values")
            t = lib().rpd_server_submit_solve_field(self.h, _ptr(x), len(x), s1 - 1, _ptr(f), C.byref(p),
                                                    _ptr(out), hv, hi, C.byref(sess))
        else:
            if grid is not None:
                self._grids.append(grid)
            t = lib().rpd_server_submit_solve_hessian(self.h, _ptr(x), len(x), grid.h if grid is not None else None,
                                                      C.byref(p), _ptr(out), hv, hi, C.byref(sess))
        if t < 0:
            raise RpdError(t, "submit solve")
        self._out[t] = (out, hb)
        return t, sess.value

    def reweight(self, session: int, w, params=None, **kw) -> int:
        """Submits a weight-only re-solve of a session; returns the ticket."""
        w = np.ascontiguousarray(w, np.float32)
        p = params if params is not None else Params.default(**kw)
        out = np.zeros((len(w), 4), np.float64)
        hb = self._hessian_buffers(len(w), p)
        t = lib().rpd_server_submit_reweight_hessian(self.h, session, _ptr(w), C.byref(p), _ptr(out),
                                                     _ptr(hb[0]) if hb else None, _ptr(hb[1]) if hb else None)
        if t < 0:
            raise RpdError(t, "submit reweight")
        self._out[t] = (out, hb)
        return t

    def wait(self, ticket: int, hessian: bool = False):
        """(moments (n,4) in user order, request info); with hessian=True
        also the Hessian rows ((n,H) areas for HC=1 or (n,H,4), ids (n,H)),
        or None when the request asked for none."""
        info = RequestInfo()
        rc = lib().rpd_server_wait(self.h, ticket, C.byref(info))
        out, hb = self._out.pop(ticket)
        if rc != RPD_OK:
            raise RpdError(rc, f"request {ticket}: {info.error.decode(errors='replace')}")
        if not hessian:
            return out, info.as_dict()
        rows = None
        if hb is not None:
            vals, ids = hb
            rows = (vals[:, :, 0] if vals.shape[2] == 1 else vals), ids
        return out, info.as_dict(), rows

    def release(self, session: int):
        rc = lib().rpd_server_release(self.h, session)
        if rc != RPD_OK:
            raise RpdError(rc, f"release session {session}")

    def bytes_in_use(self) -> int:
        return lib().rpd_server_bytes_in_use(self.h)

    def close(self):
        if self.h:
            lib().rpd_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
