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


def _split_case():
    import numpy as np
    from starlab_b200 import ics
    n = 1001
    m, x, v = ics.plummer(n, 3)
    rng = np.random.default_rng(4)
    a, j = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    idx = np.array([0, 5, 255, 256, 499, 500, 501, 767, 768, 1000])
    return n, m, x, v, a, j, idx


def _split_worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from oracle.oracle import G6Oracle
    from split_cpu import CpuSplitBackend
    from starlab_b200.dist import Dist
    from starlab_b200.distributed import SplitCluster
    d = Dist(use_cuda=False, timeout_s=60)
    n, m, x, v, a, j, idx = _split_case()
    sc = SplitCluster(d, n, block_j=256, backend=CpuSplitBackend())
    sc.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    ti = 1.0 / 128
    xp, vp = G6Oracle().predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    acc, jerk, pot, nn = sc.force(ti, idx, xp[idx], vp[idx], 1e-6)
    q.put((rank, acc, jerk, pot, nn, sc.off, sc.nl))
    d.close()


def _run_split(world):
    import torch.multiprocessing as mp
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
    return sorted(out, key=lambda o: o[0])


def test_split_cluster_bit_identical_across_world_sizes():
    """The j-split exchange (block partials -> MAX of exponents and r^2 ->
    fixed-point SUM and j MAX -> FP64) gives the same bits on 1, 2, 3 and 4
    ranks (four blocks of 256 j dealt out contiguously), and the oracle's
    single-process answer within FP64 rounding (CPU stand-in for each
    rank's kernels: tests/split_cpu.py)."""
    import numpy as np
    from oracle.oracle import G6Oracle
    runs = {w: _run_split(w) for w in (1, 2, 3, 4)}
    base = runs[1][0]
    for w, out in runs.items():
        spans = [(o[5], o[6]) for o in out]
        assert sum(c for _, c in spans) == 1001 and all(off % 256 == 0 for off, _ in spans), spans
        for o in out:
            for k in (1, 2, 3, 4):
                assert np.array_equal(np.asarray(o[k]).view(np.uint8), np.asarray(base[k]).view(np.uint8)), (w, k)
    n, m, x, v, a, j, idx = _split_case()
    orc = G6Oracle()
    xp, vp = orc.predict(1.0 / 128, 0.0, x, v, 0.5 * a, j / 6.0)
    ra, rj, rp, rn, _ = orc.force(xp, vp, m, idx, xp[idx], vp[idx], 1e-6)
    _, acc, jerk, pot, nn, _, _ = base
    assert np.allclose(acc, ra, rtol=1e-12, atol=0)
    assert np.allclose(jerk, rj, rtol=1e-11, atol=0)
    assert np.allclose(pot, rp, rtol=1e-13, atol=0)
    assert np.array_equal(nn, rn)


def test_slice_of_covers_everything():
    from starlab_b200.distributed import block_range, slice_of
    for n in (0, 1, 7, 1000, 1001):
        for w in (1, 2, 3, 8):
            spans = [slice_of(n, w, r) for r in range(w)]
            assert sum(c for _, c in spans) == n
            pos = 0
            for off, c in spans:
                assert off == pos
                pos += c
    for n in (0, 1, 255, 256, 1001, 70000):
        for w in (1, 2, 3, 8):
            pos = 0
            for r in range(w):
                off, c = block_range(n, 256, w, r)
                assert off == pos and (c == 0 or off % 256 == 0)
                pos += c
            assert pos == n

