"""One cluster's j-set split across GPUs (one process per GPU).

The reference's only distributed scheme (kira_ev.C:275-420, under -DUSEMPI)
gives every rank a contiguous range of the top-level nodes as j-particles,
computes each i's partial acc/jerk/pot over that range, and combines them
with MPI_Allreduce: SUM for the sums (kira_ev.C:327-328) and MINLOC for the
nearest neighbour (kira_ev.C:409-410).

SplitCluster keeps the whole exchange on the device and makes it
independent of the rank count:

  * the global j-set is cut into blocks of `block_j` j; rank r holds a
    contiguous run of whole blocks (`block_range`) at local addresses
    0..n_r-1 (index == address, so the engine's fast self test applies);
  * a force call computes, per block, the FP64 partial sums of the i-block
    (one split of the force kernel, computed identically on whichever rank
    holds the block) -- g6b200_split_begin, which also writes each (i,
    quantity)'s largest exponent and each i's smallest nearest-neighbour r^2;
  * all_reduce MAX of those (int64): every rank now has the same fixed-point
    scale per (i, quantity) and the global smallest r^2;
  * g6b200_split_fix converts every block partial to 64-bit fixed point on
    that scale and sums them exactly (int64), and proposes its smallest
    global j whose r^2 equals the global minimum;
  * all_reduce SUM of the fixed-point sums and MAX of the negated j (the
    first address on ties, as update_nn_coll, hdyn_inline.C:44);
  * g6b200_split_finish converts back to FP64.

Integer sums are exact and order-independent, so the results are
bit-identical for any number of ranks (given the same block size).  All
collectives are on int64 device tensors (NCCL over NVLink on GPUs; gloo on
CPU for the tests); no host round trip.

The per-rank work is behind a small backend interface (begin / fix /
finish on torch tensors), `EngineBackend` by default; tests substitute a
CPU stand-in to exercise the exchange on machines without a GPU.
"""
import ctypes

import numpy as np

BLOCK_J = 8192  # j per block (a multiple of the force kernel's tiles)


def slice_of(n, world, rank):
    """Contiguous range of a rank (the reference's decomp, kira_ev.C:135-148)."""
    base, extra = divmod(n, world)
    off = rank * base + min(rank, extra)
    return off, base + (1 if rank < extra else 0)


def block_range(n, block_j, world, rank):
    """(first global address, count) of rank's run of whole blocks: the
    blocks are dealt out contiguously, as evenly as they divide."""
    nblocks = (n + block_j - 1) // block_j
    b0, nb = slice_of(nblocks, world, rank)
    off = min(n, b0 * block_j)
    end = min(n, (b0 + nb) * block_j)
    return off, end - off


class EngineBackend:
    """Per-rank work on this rank's GPU through the C ABI (libg6b200.so)."""

    def __init__(self, cluster_id, precision, npipes, device):
        import torch
        from .g6 import G6Engine, _ptr
        self.torch = torch
        self.dev = torch.device(device)
        self.eng = G6Engine(cluster_id=cluster_id, precision=precision, npipes=npipes)
        self.lib, self.cid, self._ptr = self.eng.lib, self.eng.cid, _ptr
        P, I, D, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
        for name, res, args in (
                ("g6b200_split_begin", I, [I, I, I, P, P, P, D, I, P, P]),
                ("g6b200_split_fix", I, [I, LL, LL, P, P, P, P]),
                ("g6b200_split_finish", I, [I, LL, LL, P, P, P, P, P, P, P, P]),
                ("g6b200_set_position_range", I, [I, D])):
            f = getattr(self.lib, name)
            f.restype, f.argtypes = res, args

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _chk(self, what, rc):
        if rc:
            self.eng._err(what, rc)

    def set_position_range(self, xmax):
        self.lib.g6b200_set_position_range(self.cid, float(xmax))

    def load(self, tj, m, j6, a2, v, x):
        self.eng.set_j_particles(tj, m, j6, a2, v, x)

    def begin(self, ti, nj, local_index, xi, vi, eps2, block_j):
        ni = len(local_index)
        self.eng.set_ti(ti)
        agree = self.torch.empty(8 * ni, dtype=self.torch.int64, device=self.dev)
        idx = np.ascontiguousarray(local_index, np.int32)
        xi = np.ascontiguousarray(xi, np.float64)
        vi = np.ascontiguousarray(vi, np.float64)
        self._keep = (idx, xi, vi)
        self._chk("g6b200_split_begin", self.lib.g6b200_split_begin(
            self.cid, int(nj), ni, self._ptr(idx), self._ptr(xi), self._ptr(vi), float(eps2), int(block_j),
            ctypes.c_void_p(agree.data_ptr()), self._stream()))
        return agree

    def fix(self, nblocks, j_offset, agree):
        ni = agree.numel() // 8
        sums = self.torch.empty(7 * ni, dtype=self.torch.int64, device=self.dev)
        negj = self.torch.empty(ni, dtype=self.torch.int64, device=self.dev)
        self._chk("g6b200_split_fix", self.lib.g6b200_split_fix(
            self.cid, int(nblocks), int(j_offset), ctypes.c_void_p(agree.data_ptr()),
            ctypes.c_void_p(sums.data_ptr()), ctypes.c_void_p(negj.data_ptr()), self._stream()))
        return sums, negj

    def finish(self, nblocks, n, agree, sums, negj):
        ni = negj.numel()
        acc, jerk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
        nn = np.empty(ni, dtype=np.int32)
        self._chk("g6b200_split_finish", self.lib.g6b200_split_finish(
            self.cid, int(nblocks), int(n), ctypes.c_void_p(agree.data_ptr()), ctypes.c_void_p(sums.data_ptr()),
            ctypes.c_void_p(negj.data_ptr()), self._stream(), self._ptr(acc), self._ptr(jerk), self._ptr(pot),
            self._ptr(nn)))
        return acc, jerk, pot, nn

    def close(self):
        self.eng.close()


class SplitCluster:
    def __init__(self, dist, n, precision="fp64", cluster_id=900, block_j=BLOCK_J, backend=None, device=None):
        self.d = dist
        self.n = int(n)
        self.block_j = int(block_j)
        self.nblocks = max(1, (self.n + self.block_j - 1) // self.block_j)
        self.off, self.nl = block_range(self.n, self.block_j, dist.world, dist.rank)
        if backend is None:
            device = device or ("cuda:%d" % dist.local)
            backend = EngineBackend(cluster_id, precision, max(self.n, 1), device)
        self.be = backend

    def set_j_particles(self, tj, mass, j6, a2, v, x):
        """Global arrays in; each rank keeps (and uploads) its own slice.
        Every rank sets the same fixed-point range (the global |x| bound)."""
        s = slice(self.off, self.off + self.nl)
        n = self.n
        tj = np.broadcast_to(np.asarray(tj, np.float64), (n,))
        self.be.set_position_range(float(np.abs(np.asarray(x)).max()) if n else 0.0)
        if self.nl > 0:
            self.be.load(np.array(tj[s]), np.array(mass[s]), np.array(j6[s]), np.array(a2[s]), np.array(v[s]),
                         np.array(x[s]))

    def _all_reduce(self, t, op):
        if self.d.world > 1:
            self.d.dist.all_reduce(t, op=getattr(self.d.dist.ReduceOp, op))

    def force(self, ti, index, xi, vi, eps2):
        """acc, jerk, pot, nn (global addresses) of the i-block, on every rank."""
        index = np.asarray(index, np.int64)
        ni = index.shape[0]
        xi = np.ascontiguousarray(xi, np.float64).reshape(ni, 3)
        vi = np.ascontiguousarray(vi, np.float64).reshape(ni, 3)
        # an i outside this rank's run gets an index no local j has
        local_idx = np.where((index >= self.off) & (index < self.off + self.nl), index - self.off,
                             self.nl + 1).astype(np.int32)
        agree = self.be.begin(ti, self.nl, local_idx, xi, vi, eps2, self.block_j)
        self._all_reduce(agree, "MAX")
        sums, negj = self.be.fix(self.nblocks, self.off, agree)
        self._all_reduce(sums, "SUM")
        self._all_reduce(negj, "MAX")
        return self.be.finish(self.nblocks, self.n, agree, sums, negj)

    def close(self):
        self.be.close()
