"""The allocation-free entry point g6b200_force_noalloc, through the C ABI.

It serves callers of this library that cannot call cudaMalloc (the device
memory belongs to their own allocator or budget, or they must not pay the
device-wide synchronisation of allocation): they pass device buffers in and
out, and the j-split partial sums live in a fixed static device array.
This test plays such a caller -- its buffers come from torch's allocator --
and checks two calls in a row against the engine's regular entry points
(g6calc_firsthalf_/g6calc_lasthalf2_ in FP64 mode) within the FP64
tolerance the parity tests use, plus the rejection of sizes beyond the
static array.  The file name sorts last so that a run stopping at the first
failure has run every other test before this one.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _fn():
    from starlab_b200 import load_library
    lib = load_library()
    f = lib.g6b200_force_noalloc
    P = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, P, P, P, ctypes.c_int, P, P, P, ctypes.c_double, P, P, P, P, P]
    f.restype = ctypes.c_int
    return lib, f


def test_noalloc_matches_regular_entry_two_calls():
    import torch
    from starlab_b200 import G6Engine, ics

    torch.cuda.set_device(0)
    lib, f = _fn()
    n, eps2 = 20000, 1e-6
    m, x, v = ics.plummer(n, 314)
    z = np.zeros((n, 3))
    eng = G6Engine(cluster_id=777, precision="fp64", npipes=4096)
    eng.set_j_particles(0.0, m, z, z, v, x)
    eng.set_ti(0.0)

    def dev(a, dtype=torch.float64):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)

    xj, vj, mj = dev(x), dev(v), dev(m)
    for ni, i0 in ((1000, 0), (333, 5000)):
        idx = np.arange(i0, i0 + ni, dtype=np.int32)
        want = eng.force(n, idx, x[idx], v[idx], eps2)
        ii = dev(idx, torch.int32)
        xi, vi = dev(x[idx]), dev(v[idx])
        acc = torch.empty((ni, 3), dtype=torch.float64, device="cuda")
        jerk = torch.empty((ni, 3), dtype=torch.float64, device="cuda")
        pot = torch.empty(ni, dtype=torch.float64, device="cuda")
        nn = torch.empty(ni, dtype=torch.int32, device="cuda")
        rc = f(n, xj.data_ptr(), vj.data_ptr(), mj.data_ptr(), ni, ii.data_ptr(), xi.data_ptr(),
               vi.data_ptr(), eps2, acc.data_ptr(), jerk.data_ptr(), pot.data_ptr(), nn.data_ptr(), None)
        assert rc == 0, lib.g6b200_last_error()
        torch.cuda.synchronize()
        got = (acc.cpu().numpy(), jerk.cpu().numpy(), pot.cpu().numpy(), nn.cpu().numpy())
        ea = np.linalg.norm(got[0] - want[0], axis=1) / np.linalg.norm(want[0], axis=1)
        ej = np.linalg.norm(got[1] - want[1], axis=1) / np.linalg.norm(want[1], axis=1)
        ep = np.abs(got[2] - want[2]) / np.abs(want[2])
        assert ea.max() <= TOL and ej.max() <= TOL and ep.max() <= TOL, (ea.max(), ej.max(), ep.max())
        assert np.array_equal(got[3], want[3])
    eng.close()


def test_noalloc_rejects_sizes_beyond_the_static_array():
    lib, f = _fn()
    limit = 32768  # G6B200_NOALLOC_MAX_NI
    rc = f(10, None, None, None, limit + 1, None, None, None, 1e-6, None, None, None, None, None)
    assert rc == -1
    assert b"scratch limit" in lib.g6b200_last_error()


def test_noalloc_direct_path_no_index_and_empty_j():
    """The remaining branches, each against the engine's FP64 mode: ni at
    the limit (one j-split, results written directly, the whole array's
    bound), no index_i (no pair skipped: the engine with indices that match
    no j), and nj = 0 (zero forces, nn = 0)."""
    import torch
    from starlab_b200 import G6Engine, ics

    torch.cuda.set_device(0)
    lib, f = _fn()
    limit = 32768  # G6B200_NOALLOC_MAX_NI
    n, eps2 = 20000, 1e-6
    m, x, v = ics.plummer(n, 2718)
    z = np.zeros((n, 3))
    eng = G6Engine(cluster_id=778, precision="fp64", npipes=limit)
    eng.set_j_particles(0.0, m, z, z, v, x)
    eng.set_ti(0.0)

    def dev(a, dtype=torch.float64):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)

    def call(nj, xj, vj, mj, ni, ii, xi, vi):
        out = (torch.empty((ni, 3), dtype=torch.float64, device="cuda"),
               torch.empty((ni, 3), dtype=torch.float64, device="cuda"),
               torch.empty(ni, dtype=torch.float64, device="cuda"),
               torch.empty(ni, dtype=torch.int32, device="cuda"))
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        rc = f(nj, ptr(xj), ptr(vj), ptr(mj), ni, ptr(ii), xi.data_ptr(), vi.data_ptr(), eps2,
               *[o.data_ptr() for o in out], None)
        assert rc == 0, lib.g6b200_last_error()
        torch.cuda.synchronize()
        return tuple(o.cpu().numpy() for o in out)

    def close(got, want):
        ea = np.linalg.norm(got[0] - want[0], axis=1) / np.linalg.norm(want[0], axis=1)
        ej = np.linalg.norm(got[1] - want[1], axis=1) / np.linalg.norm(want[1], axis=1)
        ep = np.abs(got[2] - want[2]) / np.abs(want[2])
        assert ea.max() <= TOL and ej.max() <= TOL and ep.max() <= TOL, (ea.max(), ej.max(), ep.max())
        assert np.array_equal(got[3], want[3])

    xj, vj, mj = dev(x), dev(v), dev(m)
    # ni at the limit: points near the cluster's own particles, each with
    # the index of the particle it sits next to (that pair is skipped)
    rng = np.random.default_rng(3)
    sel = rng.integers(0, n, limit)
    xq = x[sel] + rng.normal(scale=1e-3, size=(limit, 3))
    vq = v[sel]
    idx = sel.astype(np.int32)
    want = eng.force(n, idx, xq, vq, eps2)
    close(call(n, xj, vj, mj, limit, dev(idx, torch.int32), dev(xq), dev(vq)), want)
    # no index_i: nothing skipped, as the engine with an index no j carries
    ni = 500
    want = eng.force(n, np.full(ni, -1, dtype=np.int32), xq[:ni], vq[:ni], eps2)
    close(call(n, xj, vj, mj, ni, None, dev(xq[:ni]), dev(vq[:ni])), want)
    # nj = 0: no j, zero sums, nn = 0
    acc, jerk, pot, nn = call(0, None, None, None, 64, None, dev(xq[:64]), dev(vq[:64]))
    assert not acc.any() and not jerk.any() and not pot.any() and not nn.any()
    eng.close()
