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
