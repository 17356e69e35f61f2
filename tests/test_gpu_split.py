"""The multi-GPU j-split's device steps (starlab_b200/csrc/split.cu through
g6b200_split_begin/fix/finish) on one GPU.

Every test here runs on one GPU, so W ranks are emulated in one process:
one engine instance per rank holds that rank's run of blocks, and the
collectives between the steps are done with torch reductions over the
ranks' device buffers (no kernels wait on one another).  The results must
be bit-identical for W = 1, 2, 3 (the fixed-point combination is exact and
order-independent) and match the FP64 oracle (the exchange over real
process groups is covered with gloo ranks in tests/test_dist.py)."""
import numpy as np
import pytest

from helpers import rel_err, rel_err_vec, snapshot

pytestmark = pytest.mark.gpu

BLOCK = 2048


def _emulated(world, mode, n, m, x, v, a, j, ti, idx, xi, vi, eps2, cid0):
    import torch
    from starlab_b200.distributed import EngineBackend, block_range
    nblocks = (n + BLOCK - 1) // BLOCK
    ranks = []
    for r in range(world):
        off, nl = block_range(n, BLOCK, world, r)
        be = EngineBackend(cid0 + r, mode, max(n, 1), "cuda:0")
        be.set_position_range(float(np.abs(x).max()))
        if nl:
            s = slice(off, off + nl)
            be.load(np.zeros(nl), m[s], j[s] / 6.0, 0.5 * a[s], v[s], x[s])
        local = np.where((idx >= off) & (idx < off + nl), idx - off, nl + 1).astype(np.int32)
        ranks.append((be, off, nl, local))
    agrees = [be.begin(ti, nl, local, xi, vi, eps2, BLOCK) for be, off, nl, local in ranks]
    agree = torch.stack(agrees).amax(0)
    fixed = [be.fix(nblocks, off, agree) for be, off, nl, local in ranks]
    sums = torch.stack([f[0] for f in fixed]).sum(0)
    negj = torch.stack([f[1] for f in fixed]).amax(0)
    outs = [be.finish(nblocks, n, agree, sums, negj) for be, off, nl, local in ranks]
    for be, *_ in ranks:
        be.close()
    for o in outs[1:]:
        for k in range(4):
            assert np.array_equal(o[k], outs[0][k])
    return outs[0]


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_split_bit_identical_across_emulated_ranks(mode, oracle):
    n = 7000  # four blocks, the last one partial
    m, x, v, a, j = snapshot(n, 21)
    ti = 1.0 / 256
    xp, vp = oracle.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    idx = np.arange(0, n, 7)
    res = {w: _emulated(w, mode, n, m, x, v, a, j, ti, idx, xp[idx], vp[idx], 1e-6, 4400 + 10 * w)
           for w in (1, 2, 3)}
    for w in (2, 3):
        for k in range(4):
            assert np.array_equal(res[w][k].view(np.uint8), res[1][k].view(np.uint8)), (w, k)
    acc, jerk, pot, nn = res[1]
    ra, rj, rp, rn, _ = oracle.force(xp, vp, m, idx, xp[idx], vp[idx], 1e-6)
    tol = 1e-12 if mode == "fp64" else 1e-6
    assert rel_err_vec(acc, ra).max() <= tol
    assert rel_err_vec(jerk, rj).max() <= (1e-12 if mode == "fp64" else 1e-5)
    assert rel_err(pot, rp).max() <= tol
    if mode == "fp64":
        assert np.array_equal(nn, rn)
    else:
        assert np.mean(nn == rn) > 0.99


def test_split_cluster_single_rank_engine(oracle):
    """SplitCluster with one rank (no process group): the default engine
    backend gives the oracle's answer."""
    from starlab_b200.dist import Dist
    from starlab_b200.distributed import SplitCluster
    n = 5000
    m, x, v, a, j = snapshot(n, 21)
    d = Dist(use_cuda=False)
    sc = SplitCluster(d, n, precision="fp64", cluster_id=4321, device="cuda:0")
    sc.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    ti = 1.0 / 256
    xp, vp = oracle.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    idx = np.arange(0, n, 37)
    acc, jerk, pot, nn = sc.force(ti, idx, xp[idx], vp[idx], 1e-6)
    ra, rj, rp, rn, _ = oracle.force(xp, vp, m, idx, xp[idx], vp[idx], 1e-6)
    assert rel_err_vec(acc, ra).max() < 1e-12
    assert rel_err_vec(jerk, rj).max() < 1e-12
    assert rel_err(pot, rp).max() < 1e-12
    assert np.array_equal(nn, rn)
    sc.close()
