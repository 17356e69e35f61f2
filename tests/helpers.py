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
