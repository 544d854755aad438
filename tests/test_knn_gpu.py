"""Device kNN parity: bit-exact lists against the oracle's exact mode
(ascending float distance, ties by stored index)."""
import numpy as np
import pytest

import oracle
from seeds_util import clustered, jittered, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


@pytest.mark.parametrize("K", [20, 50, 70])
def test_knn_uniform(rpd, K):
    x = uniform(30000, seed=K)
    kn = rpd.KNearests(x)
    assert kn.buildKnearests(K)
    got = kn.getNearests()
    want = oracle.knn(x.astype(np.float64), K, knn_mode=1)
    assert np.array_equal(got, want)


def test_knn_permutation_matches_oracle(rpd):
    x = uniform(20000, seed=5)
    kn = rpd.KNearests(x)
    dim, perm, _ = oracle.bin_seeds(x.astype(np.float64))
    assert kn._s.dim == dim
    assert np.array_equal(kn.getPermutation(), perm)


@pytest.mark.parametrize("K", [50, 105, 252])
def test_knn_lattice_and_large_k(rpd, K):
    x = jittered(25, seed=K)
    kn = rpd.KNearests(x)
    kn.buildKnearests(K)
    want = oracle.knn(x.astype(np.float64), K, knn_mode=1)
    assert np.array_equal(kn.getNearests(), want)


def test_knn_clustered(rpd):
    x = clustered(20000)
    kn = rpd.KNearests(x)
    kn.buildKnearests(50)
    want = oracle.knn(x.astype(np.float64), 50, knn_mode=1)
    assert np.array_equal(kn.getNearests(), want)


def test_knn_fewer_points_than_k(rpd):
    x = uniform(40, seed=9)
    kn = rpd.KNearests(x)
    kn.buildKnearests(50)
    got = kn.getNearests()
    want = oracle.knn(x.astype(np.float64), 50, knn_mode=1)
    assert np.array_equal(got, want)
    assert (got[:, 39:] == -1).all()


def test_knn_exact_ties_broken_by_index(rpd):
    # an exact lattice: many equal distances
    m = 20
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    x = np.zeros((len(g), 4), np.float32)
    x[:, :3] = ((g + 0.5) * 50.0).astype(np.float32)
    kn = rpd.KNearests(x)
    kn.buildKnearests(30)
    want = oracle.knn(x.astype(np.float64), 30, knn_mode=1)
    assert np.array_equal(kn.getNearests(), want)


def _lattice(m=20, h=50.0):
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    x = np.zeros((len(g), 4), np.float32)
    x[:, :3] = ((g + 0.5) * h).astype(np.float32)
    return x


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("case,K", [("uniform", 20), ("uniform", 50), ("uniform", 70), ("jittered", 105),
                                    ("jittered", 128), ("clustered", 50), ("ties", 30), ("few", 50)])
def test_knn_variants_bitexact(rpd, variant, case, K):
    """Both neighbour-search variants (a warp per seed, a thread per seed),
    pinned on the context, give the oracle's exact lists."""
    x = {"uniform": lambda: uniform(30000, seed=K), "jittered": lambda: jittered(25, seed=K),
         "clustered": lambda: clustered(20000), "ties": _lattice, "few": lambda: uniform(40, seed=9)}[case]()
    ctx = rpd.default_context()
    prev = ctx.knn_variant(K)
    try:
        assert ctx.knn_variant(K, variant) == variant
        kn = rpd.KNearests(x)
        assert kn.buildKnearests(K)
        got = kn.getNearests()
    finally:
        ctx.knn_variant(K, prev)
    want = oracle.knn(x.astype(np.float64), K, knn_mode=1)
    assert np.array_equal(got, want)


def test_knn_variant_trial_and_forcing_flags(rpd):
    """Without a pinned variant, the first search with K times both and keeps
    the faster; the launch flags force either; the solves agree bit for bit."""
    g = rpd.Grid.blob(40, 5, 2)
    x = jittered(30, seed=6, weights=True)
    ctx = rpd.default_context()
    ctx.knn_variant(37, -1)
    out = []
    for flags in (0, rpd.FLAG_KNN_WARP, rpd.FLAG_KNN_THREAD):
        s = rpd.Solver().set_points(x).set_grid(g)
        s.launch(K=37, P=30, V=40, T=100, flags=flags | rpd.FLAG_NO_PROBE)
        st = s.stats()
        out.append((s.moments().copy(), s.status().copy(), st["passes"][0]["knn_variant"]))
        s.close()
    assert ctx.knn_variant(37) in (0, 1)  # chosen by the trial
    assert out[1][2] == "warp" and out[2][2] == "thread"
    for m, st, _ in out[1:]:
        assert np.array_equal(m, out[0][0]) and np.array_equal(st, out[0][1])
