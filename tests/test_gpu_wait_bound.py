"""Failure detection on the GPU without a fault: every j-tile copy the force
kernel waits for is waited on with a time bound (mbar_wait_bounded, about a
second in the force kernel), and a wait that runs out sets a status bit that
g6calc_lasthalf2_ turns into return code 3 -- kira then resets and retries
(hdyn_grape6.C:892-899, exercised by the host-side injection in
test_gpu_kira.py).  Here the same bounded wait runs on a barrier that
nothing arrives at (g6b200_selftest_copy_timeout): it must end after its
bound with code 3 and the timeout message, and the engine must compute the
next call exactly as before.
"""
import ctypes
import time

import numpy as np
import pytest

from helpers import rel_err, rel_err_vec, snapshot

pytestmark = pytest.mark.gpu


def test_copy_wait_bound_ends_with_an_error_and_the_engine_goes_on(oracle):
    from starlab_b200 import G6Engine, load_library
    lib = load_library()
    lib.g6b200_selftest_copy_timeout.argtypes = [ctypes.c_int, ctypes.c_double]
    lib.g6b200_selftest_copy_timeout.restype = ctypes.c_int
    m, x, v, a, j = snapshot(2048, 31)
    e = G6Engine(cluster_id=71, precision="fp64", npipes=2048)
    e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    e.set_ti(0.0)
    idx = np.arange(0, 2048, 7, dtype=np.int32)
    before = e.force(2048, idx, x[idx], v[idx], 1e-6)
    t0 = time.perf_counter()
    rc = lib.g6b200_selftest_copy_timeout(71, 20.0)
    waited = time.perf_counter() - t0
    assert rc == 3
    assert b"timed out" in lib.g6b200_last_error()
    assert 0.015 < waited < 5.0            # ended by its 20 ms bound, not at once and not hung
    after = e.force(2048, idx, x[idx], v[idx], 1e-6)
    for q in range(4):
        assert np.array_equal(before[q], after[q])
    ra, rj, rp, rn, _ = oracle.force(x, v, m, idx, x[idx], v[idx], 1e-6)
    assert rel_err_vec(after[0], ra).max() < 1e-12
    assert rel_err(after[2], rp).max() < 1e-12
    e.close()
