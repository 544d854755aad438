"""The allocation-free binning entry point (rpd_bin_seeds_noalloc) against the
existing one (rpd_solver_set_points + rpd_solver_get_permutation), through the
C ABI, on calls in a row that share its static scratch.

Its callers cannot allocate device memory (they run inside another memory
pool or a host that forbids cudaMalloc after start-up), so the test owns
every buffer and the entry point must bin into them exactly as the solver
does: the same permutation, stored seeds and bin prefix sums (integers:
bit-exact)."""
import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _entry(rpd):
    f = rpd.lib().rpd_bin_seeds_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p]
    return f


def test_noalloc_binning_matches_existing_entry_point():
    import torch

    import rpd
    from rpd import synth

    rpd.default_context()
    f = _entry(rpd)
    # two calls in a row (then the first again): stale scratch of one call
    # must not leak into the next
    for n, seed in [(60000, 21), (200000, 22), (60000, 21)]:
        x = synth.uniform(n, seed)
        s = rpd.Solver().set_points(x)
        perm_ref, dim_ref = s.permutation(), s.dim
        s.close()
        xd = torch.from_numpy(x).cuda()
        stored = torch.full_like(xd, -1.0)
        perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        cap = dim_ref ** 3 + 1
        counters = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        dim = C.c_int(0)
        torch.cuda.synchronize()
        rc = f(xd.data_ptr(), n, stored.data_ptr(), perm.data_ptr(), counters.data_ptr(), cap, C.byref(dim), None)
        assert rc == rpd.RPD_OK
        assert dim.value == dim_ref
        p = perm.cpu().numpy()
        assert np.array_equal(p, perm_ref)
        assert np.array_equal(stored.cpu().numpy(), x[p])
        odim, operm, ocounters = oracle.bin_seeds(x.astype(np.float64))
        assert odim == dim_ref and np.array_equal(operm, p)
        assert np.array_equal(counters.cpu().numpy(), ocounters)


def test_noalloc_binning_on_a_caller_stream_and_its_errors():
    """On the caller's own (non-null) stream the result is the solver's; a
    counters buffer below dim^3 + 1 is RPD_ERR_INVALID with dim reported, a
    bin holding more than 4096 seeds RPD_ERR_DEGENERATE, and a NaN seed
    RPD_ERR_INVALID -- then the next call works again."""
    import torch

    import rpd
    from rpd import synth

    rpd.default_context()
    f = _entry(rpd)
    n = 100000
    x = synth.uniform(n, 31)
    s = rpd.Solver().set_points(x)
    perm_ref, dim_ref = s.permutation(), s.dim
    s.close()
    xd = torch.from_numpy(x).cuda()
    stored = torch.empty_like(xd)
    perm = torch.empty((n,), dtype=torch.int32, device="cuda")
    cap = dim_ref ** 3 + 1
    counters = torch.empty((cap,), dtype=torch.int32, device="cuda")
    dim = C.c_int(0)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    rc = f(xd.data_ptr(), n, stored.data_ptr(), perm.data_ptr(), counters.data_ptr(), cap, C.byref(dim),
           C.c_void_p(stream.cuda_stream))
    assert rc == rpd.RPD_OK and dim.value == dim_ref
    assert np.array_equal(perm.cpu().numpy(), perm_ref)
    # counters too small: rejected with dim reported, before any device work
    dim = C.c_int(0)
    rc = f(xd.data_ptr(), n, stored.data_ptr(), perm.data_ptr(), counters.data_ptr(), 1, C.byref(dim), None)
    assert rc == -1 and dim.value == dim_ref
    # 5000 seeds in one bin (bins of 1000/32 at 100K seeds): degenerate
    y = x.copy()
    y[:5000, :3] = np.random.default_rng(1).random((5000, 3), dtype=np.float32) * 20.0
    yd = torch.from_numpy(y).cuda()
    rc = f(yd.data_ptr(), n, stored.data_ptr(), perm.data_ptr(), counters.data_ptr(), cap, C.byref(dim), None)
    assert rc == -7  # RPD_ERR_DEGENERATE
    y = x.copy()
    y[123, 1] = float("nan")
    yd = torch.from_numpy(y).cuda()
    rc = f(yd.data_ptr(), n, stored.data_ptr(), perm.data_ptr(), counters.data_ptr(), cap, C.byref(dim), None)
    assert rc == -1  # RPD_ERR_INVALID
    rc = f(xd.data_ptr(), n, stored.data_ptr(), perm.data_ptr(), counters.data_ptr(), cap, C.byref(dim), None)
    assert rc == rpd.RPD_OK
    assert np.array_equal(perm.cpu().numpy(), perm_ref)


def test_noalloc_binning_rejects_too_many_seeds():
    import rpd

    f = _entry(rpd)
    dim = C.c_int(0)
    # rejected before any device work: the pointers are never dereferenced
    fake = C.c_void_p(16)
    rc = f(fake, rpd_max(rpd) + 1, fake, fake, fake, 1 << 20, C.byref(dim), None)
    assert rc == -8  # RPD_ERR_CAPACITY


def rpd_max(rpd):
    return 262144
