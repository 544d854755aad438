"""Domain grids on the host: generators, the reference text format,
validation (no GPU)."""
import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.lib()
    return m


def test_blob_is_valid_closed_and_oriented(rpd):
    g = rpd.Grid.blob(24, 5, 2)
    ok, why = g.valid(return_reason=True)
    assert ok, why
    assert g.getVolume() > 0
    a = g.arrays()
    assert set(np.unique(a["in_domain"])) <= {0, 2}
    assert a["offsets"][-1] == len(a["tri_list"])


def test_save_load_roundtrip(rpd, tmp_path):
    g = rpd.Grid.blob(16, 3, 5)
    p = tmp_path / "g.txt"
    assert g.save(p)
    h = rpd.Grid()
    assert h.load(p)
    a, b = g.arrays(), h.arrays()
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    assert abs(g.getVolume() - h.getVolume()) < 1e-6 * g.getVolume()


def test_load_rejects_bad_files(rpd, tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("2\n0 0 0 0 0 0 0 7\n")
    assert not rpd.Grid().load(p)
    assert not rpd.Grid().load(tmp_path / "missing.txt")


def test_cube_volume(rpd):
    g = rpd.Grid.cube(8)
    assert g.valid()
    assert abs(g.getVolume() - (1000 - 1000 / 8) ** 3) < 1e-3


def test_grid_from_arrays_flips_orientation(rpd):
    g = rpd.Grid.blob(12, 2, 1)
    a = g.arrays()
    t = a["triangles"][:, [1, 0, 2]]
    h = rpd.Grid.from_arrays(a["size"], a["in_domain"], a["points"], t, a["tri_list"], a["offsets"])
    assert abs(h.getVolume() - g.getVolume()) < 1e-6 * g.getVolume()


def test_oracle_fp64_volume_on_blob(rpd):
    from seeds_util import jittered

    g = rpd.Grid.blob(24, 5, 2)
    a = g.arrays()
    ga = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
    b, s = oracle.solve(jittered(16, seed=1).astype(np.float64), grid=ga, K=40, P=40, V=60, use_double=True)
    assert (s == oracle.SUCCESS).all()
    assert abs(b[:, 3].sum() / g.getVolume() - 1) < 1e-12


def test_poisson_disk_generator(rpd):
    from rpd import synth

    x = synth.poisson_disk(50_000, seed=3)
    y = synth.poisson_disk(50_000, seed=3)
    assert len(x) == 50_000 and np.array_equal(x, y)  # seeded
    assert (x[:, :3] >= 0).all() and (x[:, :3] <= 1000).all() and (x[:, 3] == 0).all()
    from scipy.spatial import cKDTree

    d, _ = cKDTree(x[:, :3].astype(np.float64)).query(x[:, :3].astype(np.float64), k=2)
    r = 0.7 * 50_000 ** (-1 / 3) * 1000
    assert d[:, 1].min() >= r * (1 - 1e-6)
