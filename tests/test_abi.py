"""The C ABI library loads without a GPU and exports every function that
include/rpd.h declares (no device calls)."""
import ctypes as C
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "rpd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(rpd_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("rpd_context_create", "rpd_solver_set_points", "rpd_solver_knn", "rpd_grid_load",
                 "rpd_solver_set_grid", "rpd_solver_launch", "rpd_solver_get_moments"):
        assert must in names


def test_library_exports_every_declared_function():
    import rpd

    lib = rpd.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_context_without_device_fails_cleanly():
    import rpd

    err = C.c_int(0)
    import torch

    if torch.cuda.is_available():
        return
    h = rpd.lib().rpd_context_create(0, C.byref(err))
    assert not h and err.value == -3


def test_params_defaults_match_reference_options():
    import rpd

    p = rpd.Params.default()
    # Options.cpp:22-28 (K 20, P 25, T 100, V 30); voronoi.cpp:1321 (5 extra passes)
    assert (p.K, p.P, p.V, p.T, p.max_extra_passes) == (20, 25, 30, 100, 5)
