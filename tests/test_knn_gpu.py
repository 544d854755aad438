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
