"""Domains built on the device (rpd_solver_set_grid_blob / _field): the
blob equals the host-built one voxel by voxel (corner flags, per-voxel
triangle counts, every triangle's vertex coordinates bit for bit, in order),
and solves on either give bitwise-equal results."""
import numpy as np
import pytest

from seeds_util import jittered

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


def triangle_coords(a):
    pts = np.asarray(a["points"], np.float32).reshape(-1, 3 if np.asarray(a["points"]).shape[-1] == 3 else 4)[:, :3]
    tri = np.asarray(a["triangles"]).reshape(-1, 3)
    lst = np.asarray(a["tri_list"])
    return pts[tri[lst]]  # (ntri, 3 corners, 3 coords) in list order


@pytest.mark.parametrize("size,seed", [(24, 2), (40, 3), (64, 7)])
def test_device_blob_equals_host_blob(rpd, size, seed):
    host = rpd.Grid.blob(size, 5, seed)
    s = rpd.Solver().set_points(jittered(4, seed=1)).set_grid_blob(size, 5, seed)
    dev = s.export_grid()
    a, b = host.arrays(), dev.arrays()
    assert int(a["size"]) == int(b["size"])
    assert np.array_equal(np.asarray(a["in_domain"]), np.asarray(b["in_domain"]))
    assert np.array_equal(np.asarray(a["offsets"]), np.asarray(b["offsets"]))
    assert np.array_equal(triangle_coords(a), triangle_coords(b))
    ok, why = dev.valid(return_reason=True)
    assert ok, why
    assert abs(dev.getVolume() - host.getVolume()) <= 1e-9 * host.getVolume()


def test_solves_on_device_and_host_blobs_are_equal(rpd):
    x = jittered(20, seed=5, weights=True)
    kw = dict(K=50, P=30, V=40, T=100)
    h = rpd.Solver().set_points(x).set_grid(rpd.Grid.blob(48, 5, 4))
    h.launch(**kw)
    d = rpd.Solver().set_points(x).set_grid_blob(48, 5, 4)
    d.launch(**kw)
    assert np.array_equal(h.status(), d.status())
    assert np.array_equal(h.moments(), d.moments())


def test_field_sphere(rpd, tmp_path):
    """A sphere of radius 0.3 from its signed distance field: a valid closed
    domain whose volume approaches 4/3 pi r^3 (reference frame), which the
    cells' masses add up to, and which saves and loads."""
    S = 48
    g = np.arange(S + 1) / S
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    f = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2) - 0.3
    s = rpd.Solver().set_points(jittered(12, seed=3)).set_grid_field(f)
    grid = s.export_grid()
    ok, why = grid.valid(return_reason=True)
    assert ok, why
    v = grid.getVolume()
    assert abs(v / (4 / 3 * np.pi * 300.0 ** 3) - 1) < 0.02
    s.launch(K=30, P=30, V=40, T=200)
    m = s.moments()
    st = s.status()
    assert (st == 4).all()
    assert abs(m[:, 3].sum() / v - 1) < 1e-6
    p = tmp_path / "sphere.txt"
    assert grid.save(p)
    again = rpd.Grid()
    assert again.load(p) and abs(again.getVolume() - v) < 1e-6 * v
