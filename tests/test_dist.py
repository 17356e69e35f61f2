"""Multi-process plumbing on CPU (gloo, world size 2).

The multi-GPU bench runs one independent cluster per rank (weak scaling, no
data-path collective): ranks must get distinct seeds, barriers must hold,
and the reported time is the maximum over ranks.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from starlab_b200.dist import Dist, cluster_seed
    d = Dist(use_cuda=False, timeout_s=60)
    d.barrier()
    mx = d.max(10.0 + rank)
    sm = d.sum(1.0)
    q.put((rank, mx, sm, cluster_seed(11, rank)))
    d.barrier()
    d.close()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [11.0, 11.0]
    assert [o[2] for o in out] == [2.0, 2.0]
    assert out[0][3] != out[1][3]


def test_weak_scaling_value():
    from starlab_b200.dist import weak_scaling_value
    # 2 ranks x 1e9 interactions x 4 steps over a slowest-rank time of 2 s
    assert weak_scaling_value(2, 1e9, 4, 2000.0) == pytest.approx(4e9)


def _split_worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import numpy as np
    from oracle.oracle import G6Oracle
    from starlab_b200 import ics
    from starlab_b200.dist import Dist
    from starlab_b200.distributed import SplitCluster
    orc = G6Oracle()

    def local_force(xj, vj, mj, local_index, xi, vi, eps2):
        acc, jerk, pot, nn, _ = orc.force(xj, vj, mj, local_index, xi, vi, eps2)
        return acc, jerk, pot, nn

    d = Dist(use_cuda=False, timeout_s=60)
    n = 1001
    m, x, v = ics.plummer(n, 3)
    rng = np.random.default_rng(4)
    a, j = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    sc = SplitCluster(d, n, local_force=local_force)
    sc.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    ti = 1.0 / 128
    xp, vp = orc.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    idx = np.array([0, 5, 499, 500, 501, 1000])
    acc, jerk, pot, nn = sc.force(ti, idx, xp[idx], vp[idx], 1e-6)
    q.put((rank, acc, jerk, pot, nn))
    d.close()


@pytest.mark.parametrize("world", [2, 3])
def test_split_cluster_exchange_matches_single_process(world):
    """j-split over ranks + SUM all-reduce + (r^2, address) minimum gives the
    single-process answer (CPU stand-in for each rank's partial sums)."""
    import numpy as np
    import torch.multiprocessing as mp
    from oracle.oracle import G6Oracle
    from starlab_b200 import ics
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    orc = G6Oracle()
    n = 1001
    m, x, v = ics.plummer(n, 3)
    rng = np.random.default_rng(4)
    a, j = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    xp, vp = orc.predict(1.0 / 128, 0.0, x, v, 0.5 * a, j / 6.0)
    idx = np.array([0, 5, 499, 500, 501, 1000])
    ra, rj, rp, rn, _ = orc.force(xp, vp, m, idx, xp[idx], vp[idx], 1e-6)
    for rank, acc, jerk, pot, nn in out:
        assert np.allclose(acc, ra, rtol=1e-12, atol=0)
        assert np.allclose(jerk, rj, rtol=1e-11, atol=0)
        assert np.allclose(pot, rp, rtol=1e-13, atol=0)
        assert np.array_equal(nn, rn)


def test_slice_of_covers_everything():
    from starlab_b200.distributed import slice_of
    for n in (0, 1, 7, 1000, 1001):
        for w in (1, 2, 3, 8):
            spans = [slice_of(n, w, r) for r in range(w)]
            assert sum(c for _, c in spans) == n
            pos = 0
            for off, c in spans:
                assert off == pos
                pos += c
