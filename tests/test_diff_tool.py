"""The result-diff figures (utils/diffResult/main.cpp:62-121) through the C
ABI and the rpd_diff tool, against a numpy restatement (no GPU)."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL = os.path.join(ROOT, "gpu-restricted-power-diagrams_b200", "rpd_diff")


def expected(a, b):
    both = (a[:, 3] > 0) & (b[:, 3] > 0)
    ba, bb = a[both, :3] / a[both, 3:], b[both, :3] / b[both, 3:]
    return {
        "sum_a": a.sum(0), "sum_b": b.sum(0), "max_mass": np.abs(b[:, 3] - a[:, 3]).max(),
        "cells_both": int(both.sum()), "max_bary": np.abs(bb - ba).max(0),
        "max_moment": np.abs(b[both, :3] - a[both, :3]).max(0),
        "avg_mass": np.abs(b[both, 3] - a[both, 3]).mean(), "avg_bary": np.abs(bb - ba).mean(0),
        "avg_moment": np.abs(b[both, :3] - a[both, :3]).mean(0),
    }


@pytest.fixture()
def pair():
    rng = np.random.default_rng(1)
    n = 500
    m = rng.uniform(0.5, 2.0, n)
    a = np.concatenate([rng.uniform(0, 1000, (n, 3)) * m[:, None], m[:, None]], 1)
    b = a + rng.normal(0, 1e-3, a.shape)
    a[7, 3] = 0.0  # a cell empty on one side: in the max mass, not in the averages
    return a, b


def check(got, want):
    for k, v in want.items():
        assert np.allclose(np.asarray(got[k], float), np.asarray(v, float), rtol=1e-12, atol=1e-15), k


def test_compare_moments_c_abi(pair):
    import rpd

    a, b = pair
    got = rpd.compare_moments(a, b)
    assert got["cells"] == len(a)
    check(got, expected(a, b))


def test_rpd_diff_tool(pair, tmp_path):
    if not os.path.exists(TOOL):
        pytest.skip("rpd_diff not built")
    a, b = pair
    paths = []
    for i, r in enumerate((a, b)):
        p = tmp_path / f"r{i}.xyzw"
        p.write_text(f"{len(r)}\n" + "\n".join(" ".join(repr(float(x)) for x in row) for row in r) + "\n")
        paths.append(str(p))
    out = subprocess.run([TOOL, "--json", *paths], capture_output=True, text=True, check=True).stdout
    check(json.loads(out), expected(a, b))
    text = subprocess.run([TOOL, *paths], capture_output=True, text=True, check=True).stdout
    assert "maximal difference by cells" in text and "average difference by cells" in text
    bad = subprocess.run([TOOL, paths[0]], capture_output=True, text=True)
    assert bad.returncode != 0
