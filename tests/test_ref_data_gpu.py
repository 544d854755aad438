"""The reference's own seed sets (data/100K-{blue,white,perturbed-grid}.xyz,
read through the library's seed loader) on the device against the FP64
oracle, at the caps the reference's README runs each with (K20/P25/V30,
K70/P30/V40, K50/P30/V40): neighbour lists bit for bit, and every cell's
status, the non-empty set, mass and barycentre (1e-5) -- in the unit cube
and restricted to a blob domain at 100^3 (the README's elephant grid is not
in the reference)."""
import numpy as np
import pytest

import oracle
import ref_data
from parity import assert_parity, compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


@pytest.fixture(scope="module")
def blob(rpd):
    g = rpd.Grid.blob(100, 5, 2)
    a = g.arrays()
    return g, oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])


@pytest.mark.parametrize("name", ref_data.NAMES)
@pytest.mark.parametrize("domain", ["cube", "blob100"])
def test_reference_data_parity(rpd, blob, name, domain):
    x = ref_data.load(name)
    caps = ref_data.CAPS[name]
    g, og = blob if domain == "blob100" else (None, None)
    s = rpd.Solver().set_points(x)
    if g is not None:
        s.set_grid(g)
    s.launch(T=100, **caps)
    got, gst = s.moments(), s.status()
    ref, rst = oracle.solve(x.astype(np.float64), grid=og, T=100, use_double=True, knn_mode=1, **caps)
    met = compare(got, gst, ref, rst)
    print(name, domain, met, s.stats()["passes"])
    assert_parity(met)
    if g is None:
        assert abs(got[:, 3].sum() / 1e9 - 1) < 1e-9
    if domain == "cube":
        # the neighbour lists of every seed, bit for bit (ties by index)
        assert np.array_equal(s.knn(caps["K"]), oracle.knn(x.astype(np.float64), caps["K"], knn_mode=1))
    s.close()
