"""The oracle: test infrastructure only.

A CPU restatement of the reference restricted-power-diagram path (see
``rpd_oracle.h`` for the function-by-function citations) plus, when it was
built here, the reference's own kernels compiled for the CPU
(``oracle/_ref/libref_kernels.so``).  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this package; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_rpd.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_kernels.so")

STATUS_NAMES = [
    "vertex_overflow", "plane_overflow", "inconsistent_boundary", "security_radius_not_reached",
    "success", "needs_exact_predicates", "empty_cell", "find_another_beginning_vertex",
    "triangle_overflow", "seed_on_border", "hessian_overflow",
]
SUCCESS = 4


class OracleGrid(C.Structure):
    _fields_ = [
        ("size", C.c_int), ("voxel_size", C.c_double), ("in_domain", C.c_void_p),
        ("points", C.c_void_p), ("npoints", C.c_int), ("triangles", C.c_void_p), ("ntri", C.c_int),
        ("tri_list", C.c_void_p), ("nlist", C.c_int), ("offsets", C.c_void_p),
    ]


class OracleParams(C.Structure):
    _fields_ = [
        ("K", C.c_int), ("P", C.c_int), ("V", C.c_int), ("T", C.c_int),
        ("vhs0", C.c_int), ("vhs1", C.c_int), ("use_double", C.c_int), ("kernels", C.c_int),
        ("knn_mode", C.c_int), ("max_extra_passes", C.c_int), ("first_pass_only", C.c_int),
        ("cube_eps", C.c_double), ("nthreads", C.c_int), ("sample_stride", C.c_int),
        ("used_cells", C.c_int), ("keep_distance", C.c_int), ("keep_volume", C.c_double),
        ("H", C.c_int), ("HC", C.c_int),
    ]


class OracleStats(C.Structure):
    _fields_ = [
        ("npasses", C.c_int), ("pass_cells", C.c_int * 8), ("pass_seconds", C.c_double * 8),
        ("final_status", C.c_int * 11), ("hs_tests", C.c_longlong), ("vertex_evals", C.c_longlong),
        ("plane_clips", C.c_longlong), ("cone_clips", C.c_longlong), ("export_vertices", C.c_longlong),
        ("knn_candidates", C.c_longlong), ("knn_seconds", C.c_double), ("cell_seconds", C.c_double),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["pass_cells"] = list(self.pass_cells)[: self.npasses]
        d["pass_seconds"] = list(self.pass_seconds)[: self.npasses]
        d["final_status"] = {STATUS_NAMES[i]: v for i, v in enumerate(self.final_status) if v}
        return d


_lib = None


def build() -> None:
    """Compiles the oracle (and the reference kernels when their sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        _lib = C.CDLL(LIB_PATH)
        _lib.oracle_solve.restype = C.c_int
        _lib.oracle_knn.restype = C.c_int
        _lib.oracle_bin.restype = C.c_int
        _lib.oracle_ref_library.restype = C.c_char_p
    return _lib


def has_reference_kernels() -> bool:
    return lib().oracle_ref_library() is not None


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class GridArrays:
    """Keeps the numpy arrays of a grid alive for an OracleGrid view."""

    def __init__(self, size, in_domain, points, triangles, tri_list, offsets):
        self.size = int(size)
        self.in_domain = np.ascontiguousarray(in_domain, dtype=np.int8)
        pts = np.asarray(points, dtype=np.float64).reshape(-1, 3 if np.asarray(points).shape[-1] == 3 else 4)
        if pts.shape[1] == 3:
            pts = np.concatenate([pts, np.zeros((len(pts), 1))], axis=1)
        self.points = np.ascontiguousarray(pts)
        self.triangles = np.ascontiguousarray(triangles, dtype=np.int32).reshape(-1)
        self.tri_list = np.ascontiguousarray(tri_list, dtype=np.int32)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        self.voxel_size = float(np.float32(1000.0) / np.float32(self.size))

    def view(self):
        return OracleGrid(
            self.size, self.voxel_size, _ptr(self.in_domain), _ptr(self.points), len(self.points),
            _ptr(self.triangles), len(self.triangles) // 3, _ptr(self.tri_list), len(self.tri_list),
            _ptr(self.offsets))


def solve(xyzw, grid=None, K=20, P=25, V=30, T=100, vhs0=2, vhs1=2, use_double=False, kernels=0,
          knn_mode=0, max_extra_passes=5, first_pass_only=False, cube_eps=None, nthreads=0,
          return_stats=False, sample_stride=1):
    """Runs the reference host flow (VoroAlgo::launch) on the CPU.

    xyzw: (n,4) seeds in the reference [0,1000]^3 frame.  Returns (bary (n,4)
    float64 = m*x, m*y, m*z, m in user order, status (n,) int32[, stats]).
    """
    x = np.ascontiguousarray(np.asarray(xyzw, dtype=np.float64).reshape(-1, 4))
    n = len(x)
    bary = np.zeros((n, 4), np.float64)
    status = np.zeros(n, np.int32)
    if cube_eps is None:
        cube_eps = 0.1 if grid is not None else 0.0
    prm = OracleParams(K, P, V, T, vhs0, vhs1, int(use_double), kernels, knn_mode, max_extra_passes,
                       int(first_pass_only), cube_eps, nthreads, sample_stride)
    st = OracleStats()
    gv = grid.view() if grid is not None else None
    rc = lib().oracle_solve(_ptr(x), n, C.byref(gv) if gv is not None else None, C.byref(prm), _ptr(bary),
                            _ptr(status), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle_solve failed: {rc}")
    return (bary, status, st.as_dict()) if return_stats else (bary, status)


def solve_hessian(xyzw, grid=None, H=50, HC=1, K=20, P=25, V=30, T=100, use_double=True, kernels=0, knn_mode=1,
                  max_extra_passes=5, cube_eps=None, nthreads=0):
    """oracle solve with --hessian (ConvexCell.cl:621-678,1133-1150): returns
    (bary, status, hess, ids) in user order; hess (n, H) areas for HC=1 or
    (n, H, 4) area-weighted facet centroids and areas for HC=4; ids (n, H)
    the facets' neighbours as user ids, -1 after a row's last facet."""
    x = np.ascontiguousarray(np.asarray(xyzw, dtype=np.float64).reshape(-1, 4))
    n = len(x)
    bary = np.zeros((n, 4), np.float64)
    status = np.zeros(n, np.int32)
    hess = np.zeros((n, H, HC), np.float64)
    ids = np.full((n, H), -1, np.int32)
    if cube_eps is None:
        cube_eps = 0.1 if grid is not None else 0.0
    prm = OracleParams(K, P, V, T, 2, 2, int(use_double), kernels, knn_mode, max_extra_passes, 0, cube_eps, nthreads,
                       1, 0, -1, 0.0, H, HC)
    gv = grid.view() if grid is not None else None
    rc = lib().oracle_solve_hessian(_ptr(x), n, C.byref(gv) if gv is not None else None, C.byref(prm), _ptr(bary),
                                    _ptr(status), _ptr(hess), _ptr(ids), None)
    if rc != 0:
        raise RuntimeError(f"oracle_solve_hessian failed: {rc}")
    return bary, status, (hess[:, :, 0] if HC == 1 else hess), ids


def solve_used(xyzw, grid, keep_distance=0, keep_volume=0.001, K=20, P=25, V=30, T=100, use_double=True, kernels=0,
               knn_mode=1, max_extra_passes=5, nthreads=0):
    """oracle solve with the reference's used cells (voronoi.cpp:1286-1393):
    returns (bary, status, used), used = per seed (user order) 0 unused, else
    its ring distance (1: used, or a face neighbour of a used cell)."""
    x = np.ascontiguousarray(np.asarray(xyzw, dtype=np.float64).reshape(-1, 4))
    n = len(x)
    bary = np.zeros((n, 4), np.float64)
    status = np.zeros(n, np.int32)
    used = np.zeros(n, np.uint8)
    prm = OracleParams(K, P, V, T, 2, 2, int(use_double), kernels, knn_mode, max_extra_passes, 0, 0.1, nthreads, 1,
                       1, keep_distance, keep_volume)
    gv = grid.view()
    rc = lib().oracle_solve_used(_ptr(x), n, C.byref(gv), C.byref(prm), _ptr(bary), _ptr(status), _ptr(used), None)
    if rc != 0:
        raise RuntimeError(f"oracle_solve_used failed: {rc}")
    return bary, status, used


def compact(bary, used, keep_distance, keep_volume, no_cell_limits=-100000.0):
    """compact_result (voronoi.cpp:583-625) in ascending user order (the
    reference's order comes from an atomic counter): the used seeds' rows, with
    w = NO_CELL_LIMITS for outer-ring cells below keep_volume.  Returns
    (rows (m,4), perm_to_user (m,))."""
    keep = np.nonzero(used)[0]
    rows = bary[keep].copy()
    border = (rows[:, 3] < keep_volume) & (used[keep] == keep_distance)
    rows[border, 3] = no_cell_limits
    return rows, keep.astype(np.int32)


def knn(xyzw, K, use_double=False, kernels=0, knn_mode=1, nthreads=0):
    """K nearest neighbours in user ids, (n,K) int32, -1 padded."""
    x = np.ascontiguousarray(np.asarray(xyzw, dtype=np.float64).reshape(-1, 4))
    out = np.zeros((len(x), K), np.int32)
    rc = lib().oracle_knn(_ptr(x), len(x), K, int(use_double), kernels, knn_mode, _ptr(out), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle_knn failed: {rc}")
    return out


def bin_seeds(xyzw, use_double=False):
    """Counting-sort binning: (dim, perm stored->user, counters)."""
    x = np.ascontiguousarray(np.asarray(xyzw, dtype=np.float64).reshape(-1, 4))
    n = len(x)
    perm = np.zeros(n, np.int32)
    dim = lib().oracle_bin(_ptr(x), n, int(use_double), _ptr(perm), None)
    counters = np.zeros(dim ** 3 + 1, np.int32)
    lib().oracle_bin(_ptr(x), n, int(use_double), _ptr(perm), _ptr(counters))
    return dim, perm, counters


def grid_invariants(grid):
    out = np.zeros(4, np.float64)
    gv = grid.view()
    lib().oracle_grid_invariants(C.byref(gv), _ptr(out))
    return out
