"""Weight-only re-solves (rpd_solver_set_weights): the same results as a
fresh solve of the re-weighted seeds, with the neighbour table reused."""
import numpy as np
import pytest

import oracle
from parity import assert_parity, compare
from seeds_util import jittered

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


def oracle_grid(g):
    a = g.arrays()
    return oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])


@pytest.mark.parametrize("with_grid", [False, True])
def test_weight_resolve_equals_fresh_solve(rpd, with_grid):
    x = jittered(24, seed=11, weights=True)
    g = rpd.Grid.blob(48, 5, 4) if with_grid else None
    kw = dict(K=50, P=30, V=40, T=100)
    s = rpd.Solver().set_points(x)
    if g is not None:
        s.set_grid(g)
    # the whole table from the start (a first launch with a domain would
    # probe and search the K nearest of the seeds near the domain only)
    s.launch(**kw, flags=rpd.FLAG_NO_PROBE)
    first_knn_ms = s.stats()["passes"][0]["knn_ms"]
    rng = np.random.default_rng(3)
    for it in range(3):
        # an optimal-transport style update of the weights
        h = 1000.0 / 24
        x[:, 3] = np.clip(x[:, 3] + rng.normal(0, 0.05 * h * h, len(x)).astype(np.float32), 0, None)
        s.set_weights(x[:, 3])
        s.launch(**kw)
        got, gst = s.moments(), s.status()
        st = s.stats()
        assert st["passes"][0]["knn_ms"] < first_knn_ms  # the neighbour table was reused
        f = rpd.Solver().set_points(x)
        if g is not None:
            f.set_grid(g)
        f.launch(**kw)
        assert np.array_equal(gst, f.status())
        assert np.array_equal(got, f.moments()), f"iteration {it}"
    ref, rst = oracle.solve(x.astype(np.float64), grid=oracle_grid(g) if g is not None else None, use_double=True,
                            knn_mode=1, **kw)
    assert_parity(compare(got, gst, ref, rst))


def test_weight_resolve_recomputes_neighbours_for_new_k(rpd):
    x = jittered(16, seed=2, weights=True)
    s = rpd.Solver().set_points(x)
    s.launch(K=20, P=30, V=40)
    s.set_weights(x[:, 3] * 0.5)
    s.launch(K=30, P=30, V=40)
    x2 = x.copy()
    x2[:, 3] *= 0.5
    f = rpd.Solver().set_points(x2)
    f.launch(K=30, P=30, V=40)
    assert np.array_equal(s.moments(), f.moments())


def test_set_weights_rejects_wrong_length(rpd):
    s = rpd.Solver().set_points(jittered(8, seed=1))
    with pytest.raises(ValueError):
        s.set_weights(np.zeros(7, np.float32))


def test_fresh_neighbours_flag_recomputes_the_table(rpd):
    x = jittered(20, seed=4, weights=True)
    s = rpd.Solver().set_points(x)
    s.launch(K=30, P=30, V=40)
    m0 = s.moments()
    s.launch(K=30, P=30, V=40)
    reused = s.stats()["passes"][0]["knn_ms"]
    s.launch(K=30, P=30, V=40, flags=rpd.FLAG_FRESH_NEIGHBOURS)
    fresh = s.stats()["passes"][0]["knn_ms"]
    assert fresh > reused
    assert np.array_equal(s.moments(), m0)


@pytest.mark.parametrize("bad", [float("nan"), float("inf"), -float("inf")])
def test_nonfinite_seeds_and_weights_rejected(rpd, bad):
    """A NaN or infinite coordinate or weight is RPD_ERR_INVALID (checked in
    the binning pass, host or device input); a rejected weight update leaves
    the seeds as they were."""
    import ctypes as C

    import torch

    x = jittered(12, seed=3, weights=True)
    for col in (0, 2, 3):
        y = x.copy()
        y[17, col] = bad
        s = rpd.Solver()
        with pytest.raises(rpd.RpdError) as e:
            s.set_points(y)
        assert e.value.code == -1 and s.n == 0
        yd = torch.from_numpy(y).cuda()
        rc = rpd.lib().rpd_solver_set_points(s.h, C.c_void_p(yd.data_ptr()), len(y), rpd.RPD_DEVICE)
        assert rc == -1 and s.n == 0
        s.set_points(x)  # the solver stays usable
        assert s.n == len(x)
        s.close()
    s = rpd.Solver().set_points(x)
    s.launch(K=20, P=30, V=40)
    m0 = s.moments().copy()
    w = x[:, 3].copy()
    w[5] = bad
    with pytest.raises(rpd.RpdError) as e:
        s.set_weights(w)
    assert e.value.code == -1
    s.launch(K=20, P=30, V=40)
    assert np.array_equal(s.moments(), m0)
