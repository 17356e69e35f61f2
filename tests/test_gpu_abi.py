"""g6 ABI conventions kira depends on, through the C ABI (GPU).

* neighbour lists overflowing the engine's per-pipe capacity: read returns
  1 and get returns 1 with nblen = max_length (hdyn_grape6.C:2081, :2319);
* npipes <= 48 (GRAPE-6 hardware convention): lists exclude i itself;
* an energy-style call (hdyn_grape6.C:1254-1305): j sent at t = 0, block
  time 0, so no prediction -- potentials equal the oracle's;
* g6_set_j_particle_ one particle at a time equals the batched upload;
* open/close/reset cycles keep working; g6_open_special picks the device.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import rel_err, rel_err_vec, snapshot

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_cid = [7000]


def eng(mode="fp64", npipes=4096):
    from starlab_b200 import G6Engine
    _cid[0] += 1
    return G6Engine(cluster_id=_cid[0], precision=mode, npipes=npipes)


def test_nb_overflow_at_engine_capacity(oracle):
    code = r"""
import sys, numpy as np
sys.path.insert(0, %r); sys.path.insert(0, %r)
from starlab_b200 import G6Engine
from helpers import snapshot
m, x, v, a, j = snapshot(3000, 5)
e = G6Engine(cluster_id=1, precision="fp64", npipes=64)
e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
e.set_ti(0.0)
c = int(np.argmin(np.sum(x * x, axis=1)))          # the most central particle
idx = np.array([c] + list(range(1000, 1007)), dtype=np.int32)
h2 = np.array([0.5 ** 2] + [1e-4] * 7)
e.calc_firsthalf(3000, idx, x[idx], v[idx], 1e-6, h2)
e.calc_lasthalf2()
rc = e.read_neighbour_list()
rc0, nb0 = e.get_neighbour_list(0, max_length=4096)
rc1, nb1 = e.get_neighbour_list(1, max_length=4096)
print(rc, rc0, len(nb0), rc1)
""" % (REPO, os.path.join(REPO, "tests"))
    env = dict(os.environ, G6B200_NBMAX="64")
    r = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    rc, rc0, n0, rc1 = map(int, r.stdout.split())
    assert rc == 1           # some list exceeded the engine's capacity
    # flagged, and nblen = max_length as the GRAPE-6 library reports an overflow
    assert rc0 == 1 and n0 == 4096
    assert rc1 == 0


def test_small_npipes_excludes_self(oracle):
    m, x, v, a, j = snapshot(2000, 8)
    e = eng(npipes=48)
    e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    e.set_ti(0.0)
    idx = np.arange(100, 140, dtype=np.int32)
    h2 = 0.1 ** 2
    e.calc_firsthalf(2000, idx, x[idx], v[idx], 1e-6, np.full(40, h2))
    e.calc_lasthalf2()
    assert e.read_neighbour_list() == 0
    want = oracle.neighbours(x, idx, x[idx], h2, include_self=False)
    for p in range(40):
        rc, nb = e.get_neighbour_list(p)
        assert rc == 0 and np.array_equal(nb, want[p])
        assert idx[p] not in nb
    e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_energy_style_call(mode, oracle):
    """All particles as i, j at t = 0, block time 0: potentials only matter."""
    m, x, v, a, j = snapshot(4096, 9)
    e = eng(mode, npipes=4096)
    e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    e.set_ti(0.0)
    idx = np.arange(4096, dtype=np.int32)
    _, _, pot, _ = e.force(4096, idx, x, v, 1e-6)
    _, _, rp, _, _ = oracle.force(x, v, m, idx, x, v, 1e-6)
    tol = 1e-12 if mode == "fp64" else 1e-6
    assert rel_err(pot, rp).max() < tol
    ep = 0.5 * np.sum(m * pot)
    assert abs(ep - 0.5 * np.sum(m * rp)) < tol * abs(ep)
    e.close()


def test_single_particle_upload_equals_batched(oracle):
    m, x, v, a, j = snapshot(700, 10)
    e1, e2 = eng(), eng()
    e1.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    for k in range(700):
        e2.set_j_particle(k, 0.0, m[k], np.zeros(3), j[k] / 6.0, 0.5 * a[k], v[k], x[k])
    ti = 1.0 / 512
    xp, vp = oracle.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    idx = np.arange(0, 700, 3, dtype=np.int32)
    for e in (e1, e2):
        e.set_ti(ti)
    r1 = e1.force(700, idx, xp[idx], vp[idx], 1e-6)
    r2 = e2.force(700, idx, xp[idx], vp[idx], 1e-6)
    for p, q in zip(r1, r2):
        assert np.array_equal(p, q)
    e1.close()
    e2.close()


def test_bulk_upload_equals_single_updates(oracle):
    """g6b200_set_j_particles of >= 4096 particles takes the bulk path
    (the caller's arrays copied straight to the device, one scatter kernel):
    permuted addresses, index != address, a repeated address (last write
    wins, as n single g6_set_j_particle_ calls), and single updates before
    and after, must leave exactly the j-memory the single calls leave."""
    n = 6001  # odd: every one of the nine gathered arrays ends off the 16-byte grid
    m, x, v, a, j = snapshot(n, 21)
    k18 = np.random.default_rng(5).normal(size=(n, 3)) * 1e-3
    rng = np.random.default_rng(4)
    perm = rng.permutation(n).astype(np.int32)
    index = perm.copy()
    index[::7] += 100000          # some ids differ from their address
    dup_addr = perm.copy()
    dup_addr[-1] = dup_addr[0]    # a repeated address: the later entry wins
    z = np.zeros(3)
    e1, e2 = eng(), eng()
    # a single update staged before the bulk upload, overwritten by it
    e1.set_j_particle(int(perm[5]), 0.0, 9.0, z, z, z, z, np.ones(3))
    e1.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x, k18=k18, address=perm, index=index)
    e1.set_j_particles(0.0, m[:10], (j / 6.0)[:10], (0.5 * a)[:10], v[:10], x[:10] * 1.01, address=perm[:10])
    e1.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x, k18=k18, address=dup_addr, index=index)
    e1.set_j_particle(int(perm[7]), 0.0, m[7], z, (j / 6.0)[7], (0.5 * a)[7], v[7], x[7] * 0.99)
    for k in range(n):
        e2.set_j_particle(int(perm[k]), 0.0, m[k], z, (j / 6.0)[k], (0.5 * a)[k], v[k], x[k], index=int(index[k]))
    e2.set_j_particle(int(dup_addr[-1]), 0.0, m[-1], z, (j / 6.0)[-1], (0.5 * a)[-1], v[-1], x[-1],
                      index=int(index[-1]))
    e2.set_j_particle(int(perm[7]), 0.0, m[7], z, (j / 6.0)[7], (0.5 * a)[7], v[7], x[7] * 0.99)
    ti = 1.0 / 512
    idx = index[:400]
    xi, vi = x[:400] + 1e-3, v[:400]
    for e in (e1, e2):
        e.set_ti(ti)
    r1 = e1.force(n, idx, xi, vi, 1e-6)
    r2 = e2.force(n, idx, xi, vi, 1e-6)
    for p, q in zip(r1, r2):
        assert np.array_equal(p, q)
    e1.close()
    e2.close()


def test_open_close_reset_cycles(oracle):
    from starlab_b200 import load_library
    lib = load_library()
    m, x, v, a, j = snapshot(500, 11)
    dev = (ctypes.c_int * 1)(0)
    assert lib.g6_open_special(1, dev) == 0
    for cycle in range(3):
        e = eng()
        e.open()
        e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
        e.set_ti(0.0)
        assert e.reset() == 0
        e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)  # reload after reset (as kira does)
        idx = np.arange(50, dtype=np.int32)
        got = e.force(500, idx, x[:50], v[:50], 1e-6)
        ref = oracle.force(x, v, m, idx, x[:50], v[:50], 1e-6)
        assert rel_err_vec(got[0], ref[0]).max() < 1e-12
        e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_small_call_path_matches_copy_path(mode):
    """Calls of <= 64 i with <= 64 staged j-updates run as one launch whose
    parameter carries the updates and i-records (no host->device copies).
    A kira-like sequence -- block updates, new block time, firsthalf /
    lasthalf2, a second chunk at the same time, a neighbour-list call --
    gives bit-identical results with that path switched off
    (G6B200_SMALL_CALLS=0), and the j-memory it leaves behind is the same."""
    import os
    from starlab_b200 import G6Engine
    n = 3000
    m, x, v, a, j = snapshot(n, 31)
    rng = np.random.default_rng(7)
    outs = []
    for small in ("1", "0"):
        os.environ["G6B200_SMALL_CALLS"] = small
        try:
            e = eng(mode, npipes=64)
        finally:
            os.environ.pop("G6B200_SMALL_CALLS", None)
        e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
        res = []
        rr = np.random.default_rng(7)
        for blk in range(12):
            upd = np.sort(rr.choice(n, 40 if blk % 3 else 64, replace=False))
            for q in upd:
                e.set_j_particle(int(q), 1e-3 * blk, m[q], np.zeros(3), (j / 6.0)[q], (0.5 * a)[q], v[q],
                                 x[q] * (1 + 1e-4 * blk))
            e.set_ti(1e-3 * (blk + 1))
            ii = np.sort(rr.choice(n, 64, replace=False)).astype(np.int32)
            res.append(e.force(n, ii, x[ii], v[ii], 1e-6))
            res.append(e.force(n, ii[:17], x[ii[:17]] * 1.0001, v[ii[:17]], 1e-6))   # same time, no updates
            h2 = np.full(9, 0.01)
            e.calc_firsthalf(n, ii[:9], x[ii[:9]], v[ii[:9]], 1e-6, h2)
            res.append(e.calc_lasthalf2())
            e.read_neighbour_list()
            res.append(tuple(e.get_neighbour_list(k) for k in range(9)))
        res.append(e.sweep(n, eps2=1e-6))   # the j-memory after all updates
        outs.append(res)
        e.close()
    def same(p, q):
        if isinstance(p, (tuple, list)):
            return len(p) == len(q) and all(same(u, w) for u, w in zip(p, q))
        return np.array_equal(np.asarray(p), np.asarray(q))

    assert len(outs[0]) == len(outs[1])
    for k, (r1, r2) in enumerate(zip(*outs)):
        assert same(r1, r2), k


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_lasthalf_without_nn_equals_lasthalf2(mode, oracle):
    """g6calc_lasthalf_ (grape6.h:68-78) returns the same acc, jerk and pot
    as g6calc_lasthalf2_ for the same call, only without the nearest
    neighbour; both agree with the oracle."""
    m, x, v, a, j = snapshot(4096, 12)
    e = eng(mode, npipes=512)
    e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    ti = 1.0 / 512
    e.set_ti(ti)
    xp, vp = oracle.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    idx = np.arange(100, 612, dtype=np.int32)
    e.calc_firsthalf(4096, idx, xp[idx], vp[idx], 1e-6)
    a1, j1, p1 = e.calc_lasthalf()
    e.calc_firsthalf(4096, idx, xp[idx], vp[idx], 1e-6)
    a2, j2, p2, nn2 = e.calc_lasthalf2()
    assert np.array_equal(a1, a2) and np.array_equal(j1, j2) and np.array_equal(p1, p2)
    ra, rj, rp, rn, _ = oracle.force(xp, vp, m, idx, xp[idx], vp[idx], 1e-6)
    tol = 1e-12 if mode == "fp64" else 1e-6
    assert rel_err_vec(a1, ra).max() <= tol and rel_err(p1, rp).max() <= tol
    e.close()
