"""Used cells and compaction on the device against the oracle (the
reference's CUSED_CELL kernels restated, FP64): the same cells kept with the
same rows, for keep distances 0 to 3, parked and inline boundary cells."""
import numpy as np
import pytest

import oracle
from parity import MASS_RTOL
from seeds_util import jittered

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


@pytest.mark.parametrize("keep_distance", [0, 1, 2, 3])
@pytest.mark.parametrize("flags", [0, 8])  # default (parked boundary cells), RPD_FLAG_NO_DEFER
def test_used_cells_match_oracle(rpd, keep_distance, flags):
    g = rpd.Grid.blob(40, 5, 2)
    a = g.arrays()
    og = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
    x = jittered(30, seed=5, weights=True)
    kw = dict(K=50, P=30, V=40, T=100)
    keep_volume = 1.0
    s = rpd.Solver().set_points(x).set_grid(g)
    s.launch(keep_distance=keep_distance, keep_volume=keep_volume, flags=flags, **kw)
    rows, ids = s.used()
    b, st, u = oracle.solve_used(x.astype(np.float64), og, keep_distance=keep_distance, keep_volume=keep_volume,
                                 use_double=True, knn_mode=1, **kw)
    ref_rows, ref_ids = oracle.compact(b, u, keep_distance, keep_volume)
    assert np.array_equal(ids, ref_ids)
    border = ref_rows[:, 3] <= -100000.0
    assert np.array_equal(rows[:, 3] <= -100000.0, border)
    # the parity bar of every cell test: 1e-5 of max(m, 1e-3), first moments
    # on the scale of the domain (1000)
    scale = np.maximum(np.abs(ref_rows[~border, 3]), 1e-3)[:, None] * np.array([1000.0, 1000.0, 1000.0, 1.0])
    assert np.max(np.abs(rows[~border] - ref_rows[~border]) / scale) < MASS_RTOL
    # the used cells alone carry the domain volume
    inner = rows[:, 3] >= keep_volume
    assert abs(rows[inner, 3].sum() / g.getVolume() - 1) < 1e-6


def test_used_cells_off_by_default(rpd):
    g = rpd.Grid.blob(24, 3, 1)
    s = rpd.Solver().set_points(jittered(12, seed=1)).set_grid(g)
    s.launch(K=30, P=30, V=40)
    with pytest.raises(rpd.RpdError):
        s.used()


@pytest.mark.parametrize("keep_distance", [0, 1])
def test_used_cells_at_negative_keep_volume(rpd, keep_distance):
    """keep_volume <= 0: every succeeding cell is used, the empty ones
    outside the domain too, and each marks the plane neighbours of its whole
    clipped cell (the early exit outside the domain is off).  At exactly 0
    the set would hang on the sign of zero masses, which the two cone
    decompositions round differently; -1 takes every cell."""
    g = rpd.Grid.blob(40, 5, 2)
    a = g.arrays()
    og = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
    x = jittered(24, seed=7, weights=True)
    kw = dict(K=50, P=30, V=40, T=100)
    s = rpd.Solver().set_points(x).set_grid(g)
    s.launch(keep_distance=keep_distance, keep_volume=-1.0, **kw)
    rows, ids = s.used()
    b, st, u = oracle.solve_used(x.astype(np.float64), og, keep_distance=keep_distance, keep_volume=-1.0,
                                 use_double=True, knn_mode=1, **kw)
    ref_rows, ref_ids = oracle.compact(b, u, keep_distance, -1.0)
    assert np.array_equal(ids, ref_ids)
    assert len(ids) == int((st == 4).sum())
    assert np.array_equal(rows[:, 3] <= -100000.0, ref_rows[:, 3] <= -100000.0)
