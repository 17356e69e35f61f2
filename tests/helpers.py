"""Shared helpers for the parity tests: snapshots and error metrics."""
import numpy as np

from starlab_b200 import ics


def rel_err_vec(a, b):
    """Per-particle |a - b| / |b| for (n, 3) arrays."""
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def rel_err(a, b):
    return np.abs(a - b) / np.abs(b)


def snapshot(n, seed, masses=None, a_scale=1.0):
    """Plummer snapshot with plausible acc/jerk for the predictor.

    acc and jerk are drawn so that the predicted displacement over the test
    step is of the order of a real Hermite step; the force tests only need
    them to be the same on both sides.
    """
    m, x, v = ics.plummer(n, seed, masses=masses)
    rng = np.random.default_rng(seed + 1000)
    a = -x / (1.0 + np.sum(x * x, axis=1, keepdims=True)) ** 1.5 * a_scale
    j = rng.normal(scale=0.5, size=(n, 3))
    return m, x, v, a, j


def oracle_forces(m, x, v, eps2, threads=None):
    """acc, jerk, pot, nn of every particle of (m, x, v) on itself from the
    FP64 oracle (oracle/g6_oracle.c), i split over host threads (the ctypes
    call releases the interpreter lock, so the chunks run in parallel)."""
    import concurrent.futures as cf
    import os
    from oracle.oracle import G6Oracle
    o = G6Oracle()
    n = len(m)
    nt = max(1, min(threads or os.cpu_count() or 1, 64))
    edges = np.linspace(0, n, 4 * nt + 1).astype(int)
    acc, jerk, pot = np.empty((n, 3)), np.empty((n, 3)), np.empty(n)
    nn = np.empty(n, dtype=np.int32)

    def chunk(k):
        i0, i1 = edges[k], edges[k + 1]
        idx = np.arange(i0, i1, dtype=np.int32)
        a, j, p, q, _ = o.force(x, v, m, idx, x[i0:i1], v[i0:i1], eps2)
        acc[i0:i1], jerk[i0:i1], pot[i0:i1], nn[i0:i1] = a, j, p, q

    with cf.ThreadPoolExecutor(nt) as ex:
        list(ex.map(chunk, range(len(edges) - 1)))
    return acc, jerk, pot, nn


def force_snapshot(n, seed, eps2, masses=None):
    """Plummer snapshot whose acc and jerk come from one FP64 oracle force
    evaluation of the snapshot itself (t_last = 0): the state a Hermite
    integrator holds after its initial force call."""
    m, x, v = ics.plummer(n, seed, masses=masses)
    a, j, _, _ = oracle_forces(m, x, v, eps2)
    return m, x, v, a, j


def near_tie_mask(xj, xi_list, nn_ref, rel=1e-6, index_i=None):
    """True where the nearest neighbour is ambiguous: the second-nearest r^2
    lies within `rel` of the nearest."""
    out = np.zeros(len(xi_list), dtype=bool)
    for k, xi in enumerate(xi_list):
        d2 = np.sum((xj - xi) ** 2, axis=1)
        if index_i is not None:
            d2[index_i[k]] = np.inf
        srt = np.partition(d2, 1)[:2]
        out[k] = srt[1] - srt[0] <= rel * srt[0]
    return out
