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

import ctypes as C
import os

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
        L.rpd_solver_create.restype = C.c_void_p
        L.rpd_solver_create.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.rpd_solver_destroy.argtypes = [C.c_void_p]
        for name in ("rpd_solver_num_points", "rpd_solver_bin_dim"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.rpd_solver_set_points.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.rpd_solver_get_permutation.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.rpd_solver_knn.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_float)]
        _lib = L
    return _lib


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Context:
    """A CUDA device bound to the engine (OpenCLContext in the reference)."""

    def __init__(self, device: int = 0):
        err = C.c_int(0)
        self.h = lib().rpd_context_create(device, C.byref(err))
        if not self.h:
            raise RpdError(err.value, f"no usable sm_100 device {device}")

    def error(self) -> str:
        return lib().rpd_context_error(self.h).decode()

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

    def set_points(self, xyzw):
        x = as_xyzw(xyzw)
        self.ctx.check(lib().rpd_solver_set_points(self.h, _ptr(x), len(x), RPD_HOST))
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
