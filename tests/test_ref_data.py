"""The reference's own seed sets (data/100K-{blue,white,perturbed-grid}.xyz)
on the CPU: the library's loader reads them as the reference's
Utils::loadSeedsFile does (Utils.cpp:36-79), and the oracle restatement
equals the reference's own kernels bit for bit on them, at the caps the
reference's README runs each with (README.md:23-25), float (the default
build, FP64 predicate) and double, without a domain and restricted to a
blob domain (the README's elephant grid is not in the reference)."""
import numpy as np
import pytest

import oracle
import ref_data


@pytest.mark.parametrize("name", ref_data.NAMES)
def test_loader_reads_reference_files(name):
    x = ref_data.load(name)
    assert x.shape == (ref_data.COUNT, 4) and x.dtype == np.float32
    lines = ref_data.text(name).decode().split("\n")
    assert int(lines[0]) == ref_data.COUNT
    want = np.array([[float(v) for v in ln.split()] for ln in lines[1:] if ln.strip()], np.float32)
    assert np.array_equal(x[:, :3], want)
    assert (x[:, 3] == 0).all()
    assert (x[:, :3] >= 0).all() and (x[:, :3] <= 1000).all()


def test_binary_seed_files_roundtrip(tmp_path):
    import rpd

    x = ref_data.load("blue")
    x[:, 3] = np.arange(len(x), dtype=np.float32)
    p = tmp_path / "seeds.bin"
    rpd.save_seeds_binary(p, x)
    assert p.stat().st_size == 8 + 16 * len(x)  # size_t count + 4 floats per seed (Utils.cpp:99-113)
    assert np.array_equal(rpd.load_seeds(p, binary=True), x)


def test_loader_rejects_bad_files(tmp_path):
    import rpd

    p = tmp_path / "short.xyz"
    p.write_text("3\n1 2 3\n4 5 6\n")
    with pytest.raises(rpd.RpdError):
        rpd.load_seeds(p)
    p.write_text("1\n1 2 x\n")
    with pytest.raises(rpd.RpdError):
        rpd.load_seeds(p)
    with pytest.raises(rpd.RpdError):
        rpd.load_seeds(tmp_path / "missing.xyz")
    p.write_text("2\n1 2 3\nnan 5 6\n")
    with pytest.raises(rpd.RpdError):
        rpd.load_seeds(p)
    p.write_text("1\n1 2 3 inf\n")
    with pytest.raises(rpd.RpdError):
        rpd.load_seeds(p, points4d=True)
    q = tmp_path / "w.xyz"
    q.write_text("2\n1 2 3 4\n5 6 7 8\n")
    assert np.array_equal(rpd.load_seeds(q, points4d=True), np.array([[1, 2, 3, 4], [5, 6, 7, 8]], np.float32))


@pytest.mark.skipif(not oracle.has_reference_kernels(), reason="reference kernels not built here")
@pytest.mark.parametrize("use_double", [0, 1])
@pytest.mark.parametrize("name", ref_data.NAMES)
def test_restatement_bitexact_with_reference_kernels(name, use_double):
    x = ref_data.load(name).astype(np.float64)
    b1, s1 = oracle.solve(x, kernels=1, use_double=use_double, **ref_data.CAPS[name])
    b0, s0 = oracle.solve(x, kernels=0, use_double=use_double, **ref_data.CAPS[name])
    assert np.array_equal(s0, s1)
    assert np.array_equal(b0, b1)
    assert (s0 == oracle.SUCCESS).all()
    assert abs(b0[:, 3].sum() / 1e9 - 1) < (1e-6 if not use_double else 1e-12)


@pytest.mark.skipif(not oracle.has_reference_kernels(), reason="reference kernels not built here")
def test_restatement_bitexact_with_reference_kernels_in_a_domain():
    import rpd

    g = rpd.Grid.blob(100, 5, 2)
    a = g.arrays()
    ga = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
    x = ref_data.load("blue").astype(np.float64)
    kw = dict(grid=ga, T=100, use_double=True, **ref_data.CAPS["blue"])
    b1, s1 = oracle.solve(x, kernels=1, **kw)
    b0, s0 = oracle.solve(x, kernels=0, **kw)
    assert np.array_equal(s0, s1)
    assert np.array_equal(b0, b1)
    ok = s0 == oracle.SUCCESS
    assert ok.mean() > 0.999
    assert abs(b0[ok, 3].sum() / g.getVolume() - 1) < 1e-6
