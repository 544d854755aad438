"""The command-line driver (rpd_voronoi, the reference test_voronoi's
options) end to end: seed and grid files in the reference formats, the
`mg` output equal to the library's moments, --hessian accepted, and the
result compared with rpd_diff."""
import json
import os
import subprocess

import numpy as np
import pytest

from seeds_util import jittered

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-restricted-power-diagrams_b200")
CLI = os.path.join(PKG, "rpd_voronoi")
DIFF = os.path.join(PKG, "rpd_diff")


def read_rows(path):
    lines = [ln for ln in open(path).read().splitlines() if ln.strip()]
    n = int(lines[0])
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]], np.float64)
    assert rows.shape == (n, 4)
    return rows


@pytest.mark.skipif(not os.path.exists(CLI), reason="rpd_voronoi not built")
def test_rpd_voronoi_mg_output_equals_library(tmp_path):
    import rpd

    x = jittered(16, seed=7, weights=True)
    seeds = tmp_path / "seeds.xyz"
    seeds.write_text(f"{len(x)}\n" + "\n".join(" ".join(f"{float(v):.9g}" for v in r) for r in x) + "\n")
    g = rpd.Grid.blob(40, 5, 3)
    gfile = tmp_path / "grid.txt"
    assert g.save(gfile)
    cmd = [CLI, "--K=30", "--P=30", "--V=40", "--T=100", f"--grid={gfile}", "--points4D", "--keepDist2=-1",
           "--output=mg", "--hessian", "--H=40", str(seeds)]
    r = subprocess.run(cmd, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = read_rows(tmp_path / "gridGPU_mg.xyzw")
    # the library on the same seeds and the loaded grid; the mg output zeroes
    # cells with a mass at most keepVolume (1, the driver's default)
    h = rpd.Grid()
    assert h.load(gfile)
    s = rpd.Solver().set_points(x).set_grid(h)
    s.launch(K=30, P=30, V=40, T=100, hessian_h=40)
    want = s.moments()
    want[want[:, 3] <= 1.0] = 0.0
    assert np.array_equal(got, want)
    ref = tmp_path / "lib.xyzw"
    ref.write_text(f"{len(want)}\n" + "\n".join(" ".join(repr(float(v)) for v in r) for r in want) + "\n")
    if os.path.exists(DIFF):
        d = json.loads(subprocess.run([DIFF, "--json", str(ref), str(tmp_path / "gridGPU_mg.xyzw")],
                                      capture_output=True, text=True, check=True).stdout)
        assert d["max_mass"] == 0.0 and d["cells"] == len(x)
