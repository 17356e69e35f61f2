"""CPU stand-in for one rank's share of the multi-GPU j-split (test
infrastructure): the FP64 oracle computes each block's partial sums, and the
three device steps of starlab_b200/csrc/split.cu (agree, fix, finish) are
restated in numpy with the same integer arithmetic, on torch CPU tensors the
gloo collectives reduce.  Lets the exchange in
starlab_b200.distributed.SplitCluster run on machines without a GPU."""
import numpy as np

NO_EXP = -(1 << 40)


def _exp(x):
    _, e = np.frexp(x)
    return np.where(x == 0.0, NO_EXP, e.astype(np.int64))


def _log2_blocks(nblocks):
    g = 0
    while (1 << g) < nblocks:
        g += 1
    return g


class CpuSplitBackend:
    def __init__(self):
        from oracle.oracle import G6Oracle
        self.o = G6Oracle()
        self.state = None

    def set_position_range(self, xmax):
        pass

    def load(self, tj, m, j6, a2, v, x):
        self.state = dict(tj=tj, m=m, j6=j6, a2=a2, v=v, x=x)

    def begin(self, ti, nj, local_index, xi, vi, eps2, block_j):
        import torch
        ni = len(local_index)
        parts = []  # per block: (q[7, ni], nn_r2[ni], nn_local[ni])
        if nj > 0:
            st = self.state
            xp, vp = self.o.predict(ti, st["tj"], st["x"], st["v"], st["a2"], st["j6"])
            for b0 in range(0, nj, block_j):
                b1 = min(nj, b0 + block_j)
                jidx = np.arange(b0, b1, dtype=np.int32)
                acc, jerk, pot, nn, r2 = self.o.force(xp[b0:b1], vp[b0:b1], st["m"][b0:b1], local_index, xi, vi,
                                                      eps2, jindex=jidx)
                q = np.concatenate([acc.T, jerk.T, pot[None]], axis=0)
                parts.append((q, r2, np.where(np.isfinite(r2), nn + b0, -1)))
        else:
            parts.append((np.zeros((7, ni)), np.full(ni, np.inf), np.full(ni, -1)))
        self.parts = parts
        e = np.full((7, ni), NO_EXP, dtype=np.int64)
        r2 = np.full(ni, np.inf)
        for q, pr2, pj in parts:
            e = np.maximum(e, _exp(q))
            r2 = np.where((pj >= 0) & (pr2 < r2), pr2, r2)
        agree = np.concatenate([e.ravel(), -r2.view(np.int64)])
        return torch.from_numpy(agree)

    def fix(self, nblocks, j_offset, agree):
        import torch
        a = agree.numpy()
        ni = a.size // 8
        e = a[:7 * ni].reshape(7, ni)
        g = _log2_blocks(nblocks)
        sc = np.where(e == NO_EXP, 0, 62 - g - e)
        r2min = (-a[7 * ni:]).view(np.float64)
        sums = np.zeros((7, ni), dtype=np.int64)
        best = np.full(ni, np.iinfo(np.int64).max, dtype=np.int64)
        for q, pr2, pj in self.parts:
            sums += np.rint(np.ldexp(q, sc)).astype(np.int64)
            hit = (pj >= 0) & (pr2 == r2min)
            best = np.where(hit, np.minimum(best, pj + j_offset), best)
        return torch.from_numpy(sums.ravel().copy()), torch.from_numpy(-best)

    def finish(self, nblocks, n, agree, sums, negj):
        a = agree.numpy()
        ni = negj.numel()
        e = a[:7 * ni].reshape(7, ni)
        g = _log2_blocks(nblocks)
        sc = np.where(e == NO_EXP, 0, 62 - g - e)
        v = np.where(e == NO_EXP, 0.0, np.ldexp(sums.numpy().reshape(7, ni).astype(np.float64), -sc))
        j = -negj.numpy()
        nn = np.where((j < 0) | (j >= n), 0, j).astype(np.int32)
        return v[0:3].T.copy(), v[3:6].T.copy(), v[6].copy(), nn

    def close(self):
        pass
