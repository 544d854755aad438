"""The device path against the golden fixtures of the reference's kernels
(FP64 build), through the C ABI."""
import glob
import os

import numpy as np
import pytest

from parity import assert_parity, compare
from test_golden import GOLDEN, load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_device_matches_reference_fp64(path):
    import rpd

    d, _ = load(path)
    K, P, V, T = (int(v) for v in d["caps"])
    s = rpd.Solver().set_points(d["xyzw"])
    if "grid_size" in d:
        s.set_grid(rpd.Grid.from_arrays(int(d["grid_size"]), d["grid_in_domain"], d["grid_points"],
                                        d["grid_triangles"], d["grid_tri_list"], d["grid_offsets"]))
    s.launch(K=K, P=P, V=V, T=T)
    met = compare(s.moments(), s.status(), d["bary_f64"], d["status_f64"])
    print(os.path.basename(path), met)
    assert_parity(met)
