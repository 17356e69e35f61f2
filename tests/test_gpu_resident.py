"""The device-resident serving loop (g6b200_res_*, starlab_b200/csrc/
resident.cu) through the C ABI.

* results equal the oracle's within the mixed-mode tolerance, and a call's
  results are bit-identical alone and gathered into one batch with other
  clusters' calls (the batch number and size returned with each call show
  they shared it), and equal the launch-per-batch server's;
* the kernel leaves after its idle time and the next submit starts it again;
* a grid barrier whose bound runs out (CTA 0 made to leave without arriving:
  no GPU fault) ends the loop with an error, the call it held fails with
  code 2, and the following calls are served normally.
"""
import time

import numpy as np
import pytest

from helpers import rel_err, rel_err_vec, snapshot

pytestmark = pytest.mark.gpu

EPS2 = 1e-6


def load(srv, n, seed):
    m, x, v, a, j = snapshot(n, seed)
    c = srv.open_cluster(n, EPS2)
    srv.set_j(c, 0.0, m, j / 6.0, 0.5 * a, v, x)
    return c, (m, x, v, a, j)


def test_resident_alone_equals_batched_and_matches_oracle(oracle):
    from starlab_b200.server import ResidentServer, Server
    srv = ResidentServer(precision="mixed")
    ids = [load(srv, n, 40 + k) for k, n in enumerate((3000, 700, 5000, 1500))]
    ti = 1.0 / 64
    c0, (m, x, v, a, j) = ids[0]
    xp, vp = oracle.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    idx = np.arange(10, 300, dtype=np.int32)
    alone = srv.wait_batch(srv.submit(c0, ti, len(m), idx, xp[idx], vp[idx]))
    assert alone[6] == 1
    srv.hold(True)
    reqs = []
    for c, (mm, xx, vv, aa, jj) in ids[1:]:
        xq, vq = oracle.predict(ti, 0.0, xx, vv, 0.5 * aa, jj / 6.0)
        k = np.arange(0, len(mm), 3, dtype=np.int32)
        reqs.append((srv.submit(c, ti, len(mm), k, xq[k], vq[k]), k, xq, vq, mm))
    rmix = srv.submit(c0, ti, len(m), idx, xp[idx], vp[idx])
    srv.hold(False)
    mixed = srv.wait_batch(rmix)
    assert mixed[6] == 1 + len(reqs), mixed[5:]
    for q in range(4):
        assert np.array_equal(alone[q], mixed[q])
    ra, rj, rp, rn, _ = oracle.force(xp, vp, m, idx, xp[idx], vp[idx], EPS2)
    assert rel_err_vec(alone[0], ra).max() < 1e-6
    assert rel_err_vec(alone[1], rj).max() < 1e-5
    assert rel_err(alone[2], rp).max() < 1e-6
    for rid, k, xq, vq, mm in reqs:
        got = srv.wait_batch(rid)
        assert got[5] == mixed[5]
        sub = k[::50]
        ra, rj, rp, rn, _ = oracle.force(xq, vq, mm, sub, xq[sub], vq[sub], EPS2)
        assert rel_err_vec(got[0][::50], ra).max() < 1e-6
    st = srv.stats()
    assert st["calls"] == 2 + len(reqs) and st["max_batch"] == 1 + len(reqs)
    srv.close()
    # the launch-per-batch server gives the same bits for the same call
    lane = Server(precision="mixed")
    c, _ = load(lane, 3000, 40)
    want = lane.wait(lane.submit(c, ti, 3000, idx, xp[idx], vp[idx]))
    lane.close()
    for q in range(4):
        assert np.array_equal(alone[q], want[q])


def test_resident_idle_exit_and_relaunch():
    import os
    from starlab_b200.server import ResidentServer
    srv = ResidentServer(precision="fp64")
    c, (m, x, v, a, j) = load(srv, 2000, 7)
    idx = np.arange(0, 2000, 5, dtype=np.int32)
    first = srv.wait(srv.submit(c, 0.0, 2000, idx, x[idx], v[idx]))
    time.sleep(0.2)  # well past the 20 ms idle time: the kernel has left
    second = srv.wait(srv.submit(c, 0.0, 2000, idx, x[idx], v[idx]))
    for q in range(4):
        assert np.array_equal(first[q], second[q])
    assert srv.stats()["launches"] >= 2
    srv.close()


def test_resident_bounded_barrier_reports_and_recovers():
    from starlab_b200 import G6Error
    from starlab_b200.server import ResidentServer
    srv = ResidentServer(precision="mixed")
    c, (m, x, v, a, j) = load(srv, 2000, 8)
    idx = np.arange(0, 500, dtype=np.int32)
    ok = srv.wait(srv.submit(c, 0.0, 2000, idx, x[idx], v[idx]))
    srv.selftest_stall()
    t0 = time.time()
    with pytest.raises(G6Error) as ei:
        srv.wait(srv.submit(c, 0.0, 2000, idx, x[idx], v[idx]))
    assert ei.value.code == 2
    assert time.time() - t0 < 30  # the barrier's bound (2 s), not a hang
    again = srv.wait(srv.submit(c, 0.0, 2000, idx, x[idx], v[idx]))
    for q in range(4):
        assert np.array_equal(ok[q], again[q])
    st = srv.stats()
    assert st["recoveries"] >= 1
    srv.close()
