"""SplitCluster on one GPU (world size 1): the per-rank engine path of the
multi-GPU j-split gives the oracle's answer (the exchange itself is covered
with gloo ranks in tests/test_dist.py)."""
import numpy as np
import pytest

from helpers import rel_err, rel_err_vec, snapshot

pytestmark = pytest.mark.gpu


def test_split_cluster_single_rank_engine(oracle):
    from starlab_b200.dist import Dist
    from starlab_b200.distributed import SplitCluster
    n = 5000
    m, x, v, a, j = snapshot(n, 21)
    d = Dist(use_cuda=False)
    sc = SplitCluster(d, n, precision="fp64", cluster_id=4321)
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
