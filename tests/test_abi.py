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


STRUCTS = {"Params": "rpd_params", "Stats": "rpd_stats", "RequestInfo": "rpd_request_info",
           "MomentDiff": "rpd_moment_diff", "BatchStats": "rpd_batch_stats"}


def test_python_structures_match_the_header(tmp_path):
    """Every ctypes mirror of an rpd.h structure has the C layout: the same
    size and the same offset for every field (a C program built against the
    header prints them)."""
    import shutil
    import subprocess

    import pytest

    import rpd

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rpd.h"', "int main(void) {"]
    for py, c in STRUCTS.items():
        cls = getattr(rpd, py)
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in cls._fields_:
            lines.append(f'  printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    bad = []
    for ln in out:
        if not ln:
            continue
        py, name, val = ln.split()
        cls = getattr(rpd, py)
        got = C.sizeof(cls) if name == "size" else getattr(cls, name).offset
        if got != int(val):
            bad.append((py, name, got, int(val)))
    assert not bad, bad


def test_cpp_facade_compiles_and_its_grid_runs_without_a_gpu(tmp_path):
    """include/rpd.hpp, the C++ facade with the reference's class names, as a
    user of the reference would call it: the whole header compiles and links
    against librpd.so; the host-side Grid part runs without a GPU."""
    import shutil
    import subprocess

    import pytest

    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    pkg = os.path.join(ROOT, "gpu-restricted-power-diagrams_b200")
    src = tmp_path / "facade.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cstring>
#include <iostream>
#include "rpd.hpp"

// the reference's driver flow (test_voronoi.cpp): compiled, run only with a GPU
static int solve(std::vector<float> const &xyzw, rpd::Grid const &grid) {
  auto ctx = rpd::Context::create(0);
  if (!ctx) return 1;
  rpd::VoroAlgo algo(ctx);
  algo.m_K = 50; algo.m_P = 30; algo.m_V = 40; algo.m_T = 100;
  algo.setInputPoints(xyzw);
  algo.setGrid(grid);
  std::vector<double> bary;
  std::vector<rpd::VoroAlgoStat> stats;
  algo.launch([&](rpd::VoroAlgo const &a) { bary = a.getBarycenters(); return true; }, stats);
  rpd::KNearests kn(ctx, xyzw);
  double t = 0;
  kn.buildKnearests(20, t);
  return bary.empty() ? 1 : 0;
}

int main(int argc, char **argv) {
  auto grid = rpd::Grid::blob(24, 3, 1);
  if (!grid || !grid->valid()) return 2;
  grid->printInvariants(std::cout);
  std::printf("volume %.6f\n", grid->getVolume());
  if (argc > 1 && std::strcmp(argv[1], "solve") == 0) return solve(std::vector<float>(4000, 1.f), *grid);
  return 0;
}
''')
    exe = tmp_path / "facade"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", pkg, "-lrpd", f"-Wl,-rpath,{pkg}"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    vol = float(out.split("volume")[-1])
    assert 1e6 < vol < 1e9
