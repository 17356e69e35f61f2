"""One cluster's j-set split across GPUs (one process per GPU).

The reference's only distributed scheme (kira_ev.C:275-420, under -DUSEMPI)
gives every rank a contiguous range of the top-level nodes as j-particles,
computes each i's partial acc/jerk/pot over that range, and combines them
with MPI_Allreduce: SUM for the sums (kira_ev.C:327-328) and MINLOC for the
nearest neighbour (kira_ev.C:409-410).  SplitCluster does the same with
one engine per rank and torch.distributed (NCCL over NVLink on GPUs, gloo
on CPU):

  * rank r holds j-addresses [off_r, off_r + n_r) at local addresses
    0..n_r-1 (index == address, so the engine's fast self test applies);
  * a force call evaluates the i-block against the local slice (an i
    outside the slice gets an index no local j has);
  * acc, jerk and pot (FP64) are summed over ranks with one all_reduce;
  * each rank's nearest-neighbour candidate is scored by its r^2 (FP64, the
    j predicted to the block time), candidates are all-gathered and every
    rank keeps the smallest (r^2, global address) -- first address on ties,
    as update_nn_coll (hdyn_inline.C:44) does.

`local_force(xj, vj, mj, local_index, xi, vi, eps2)` may replace the GPU
engine for the per-rank partial sums (used on machines without a GPU to
test the exchange).
"""
import numpy as np


def slice_of(n, world, rank):
    """Contiguous j-range of a rank (the reference's decomp, kira_ev.C:135-148)."""
    base, extra = divmod(n, world)
    off = rank * base + min(rank, extra)
    return off, base + (1 if rank < extra else 0)


class SplitCluster:
    def __init__(self, dist, n, precision="fp64", cluster_id=900, local_force=None, device="cpu"):
        self.d = dist
        self.n = int(n)
        self.off, self.nl = slice_of(self.n, dist.world, dist.rank)
        self.local_force = local_force
        self.device = device
        self.eng = None
        if local_force is None:
            from .g6 import G6Engine
            self.eng = G6Engine(cluster_id=cluster_id, precision=precision, npipes=max(self.n, 1))
        self.state = None

    def set_j_particles(self, tj, mass, j6, a2, v, x):
        """Global arrays in; each rank keeps (and uploads) its own slice."""
        s = slice(self.off, self.off + self.nl)
        n = self.n
        tj = np.broadcast_to(np.asarray(tj, np.float64), (n,))
        self.state = dict(tj=np.array(tj[s]), m=np.array(mass[s]), j6=np.array(j6[s]), a2=np.array(a2[s]),
                          v=np.array(v[s]), x=np.array(x[s]))
        if self.eng is not None and self.nl > 0:
            st = self.state
            self.eng.set_j_particles(st["tj"], st["m"], st["j6"], st["a2"], st["v"], st["x"])

    def _predict_local(self, ti):
        st = self.state
        dt = (ti - st["tj"])[:, None]
        xp = st["x"] + dt * (st["v"] + dt * (st["a2"] + dt * st["j6"]))
        vp = st["v"] + dt * (2.0 * st["a2"] + dt * (3.0 * st["j6"]))
        return xp, vp

    def force(self, ti, index, xi, vi, eps2):
        """acc, jerk, pot, nn (global addresses) of the i-block, on every rank."""
        import torch
        index = np.asarray(index, np.int64)
        ni = index.shape[0]
        xi = np.ascontiguousarray(xi, np.float64).reshape(ni, 3)
        vi = np.ascontiguousarray(vi, np.float64).reshape(ni, 3)
        local_idx = np.where((index >= self.off) & (index < self.off + self.nl), index - self.off,
                             self.nl + 1).astype(np.int32)
        if self.nl == 0:
            acc, jerk, pot = np.zeros((ni, 3)), np.zeros((ni, 3)), np.zeros(ni)
            nn = np.full(ni, -1, np.int64)
        elif self.local_force is not None:
            xp, vp = self._predict_local(ti)
            acc, jerk, pot, nn = self.local_force(xp, vp, self.state["m"], local_idx, xi, vi, eps2)
            nn = np.asarray(nn, np.int64)
        else:
            self.eng.set_ti(ti)
            acc, jerk, pot, nn = self.eng.force(self.nl, local_idx, xi, vi, eps2)
            nn = np.asarray(nn, np.int64)
        # score the local nn candidate in FP64 (excluding i itself / empty)
        r2 = np.full(ni, np.inf)
        gj = np.full(ni, np.iinfo(np.int64).max, np.int64)
        if self.nl > 0:
            xp, _ = self._predict_local(ti)
            ok = (nn >= 0) & (nn < self.nl) & (nn != local_idx)
            d = xp[np.clip(nn, 0, self.nl - 1)] - xi
            r2 = np.where(ok, np.sum(d * d, axis=1), np.inf)
            gj = np.where(ok, nn + self.off, np.iinfo(np.int64).max)
        dev = self.device
        sums = torch.from_numpy(np.concatenate([acc.ravel(), jerk.ravel(), pot])).to(dev)
        if self.d.world > 1:
            self.d.dist.all_reduce(sums, op=self.d.dist.ReduceOp.SUM)
            cand_r2 = [torch.empty(ni, dtype=torch.float64, device=dev) for _ in range(self.d.world)]
            cand_j = [torch.empty(ni, dtype=torch.int64, device=dev) for _ in range(self.d.world)]
            self.d.dist.all_gather(cand_r2, torch.from_numpy(r2).to(dev))
            self.d.dist.all_gather(cand_j, torch.from_numpy(gj).to(dev))
            r2s = np.stack([c.cpu().numpy() for c in cand_r2])
            js = np.stack([c.cpu().numpy() for c in cand_j])
        else:
            r2s, js = r2[None], gj[None]
        sums = sums.cpu().numpy()
        acc = sums[:3 * ni].reshape(ni, 3)
        jerk = sums[3 * ni:6 * ni].reshape(ni, 3)
        pot = sums[6 * ni:]
        # lexicographic minimum over ranks of (r^2, address)
        order = np.lexsort((js, r2s), axis=0)[0]
        best_j = js[order, np.arange(ni)]
        nn = np.where(best_j == np.iinfo(np.int64).max, 0, best_j).astype(np.int32)
        return acc, jerk, pot, nn

    def close(self):
        if self.eng is not None:
            self.eng.close()
