"""Served-stream workload: force calls from many clusters arriving as a
Poisson process, run through the batching server or through the plain
engine one call at a time.

Clusters: N log-uniform in [n_lo, n_hi] (seeded Plummer spheres, equal
masses); calls: Poisson arrivals at `rate` per second, each for a uniformly
chosen cluster, with an i-block of ni particles drawn from p(ni) ~ 1/ni on
[1, N] (a power law of slope -1) starting at a random address.  Each call
carries a new block time, so the cluster's j-set is predicted again.
"""
import queue
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import ics

EPS2 = 1e-6


def make_clusters(k, seed, n_lo=512, n_hi=65536):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), k)).astype(int)
    out = []
    for c, n in enumerate(ns):
        m, x, v = ics.plummer(int(n), seed * 1000 + c)
        a = -x / (1.0 + np.sum(x * x, axis=1, keepdims=True)) ** 1.5
        j = np.zeros_like(x)
        out.append((m, x, v, a, j))
    return out


def make_stream(clusters, rate, n_calls, seed):
    rng = np.random.default_rng(seed + 1)
    t = np.cumsum(rng.exponential(1.0 / rate, n_calls))
    calls = []
    for q in range(n_calls):
        c = int(rng.integers(0, len(clusters)))
        n = len(clusters[c][0])
        ni = int(min(n, max(1, np.exp(rng.uniform(0, np.log(n))))))
        i0 = int(rng.integers(0, n - ni + 1))
        calls.append((float(t[q]), c, ni, i0, 1e-6 * (q + 1)))
    return calls


def _inputs(cl, ni, i0, ti):
    m, x, v, a, j = cl
    h = ti
    xs = x[i0:i0 + ni] + h * (v[i0:i0 + ni] + h * 0.5 * a[i0:i0 + ni])
    vs = v[i0:i0 + ni] + h * a[i0:i0 + ni]
    return np.arange(i0, i0 + ni, dtype=np.int32), xs, vs


def run_served(server, clusters, calls):
    ids = []
    for (m, x, v, a, j) in clusters:
        c = server.open_cluster(len(m), EPS2)
        server.set_j(c, 0.0, m, j / 6.0, 0.5 * a, v, x)
        ids.append(c)
    pre = [_inputs(clusters[c], ni, i0, ti) for (_, c, ni, i0, ti) in calls]
    lat = [None] * len(calls)
    pool = ThreadPoolExecutor(max_workers=64)
    futs = []
    t0 = time.perf_counter()
    for q, (ta, c, ni, i0, ti) in enumerate(calls):
        while True:
            dt = t0 + ta - time.perf_counter()
            if dt <= 0:
                break
            time.sleep(min(dt, 0.0005))
        idx, xs, vs = pre[q]
        rid = server.submit(ids[c], ti, len(clusters[c][0]), idx, xs, vs)
        futs.append((q, pool.submit(server.wait, rid)))
    for q, f in futs:
        lat[q] = f.result()[4]
    wall = time.perf_counter() - t0
    pool.shutdown()
    inter = sum(ni * len(clusters[c][0]) for (_, c, ni, _, _) in calls)
    return np.array(lat), wall, inter


def run_sequential(make_engine, clusters, calls):
    """The plain engine serving the same stream one call at a time (FIFO)."""
    engs = []
    for k, (m, x, v, a, j) in enumerate(clusters):
        e = make_engine(k, len(m))
        e.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
        engs.append(e)
    pre = [_inputs(clusters[c], ni, i0, ti) for (_, c, ni, i0, ti) in calls]
    lat = np.empty(len(calls))
    t0 = time.perf_counter()
    for q, (ta, c, ni, i0, ti) in enumerate(calls):
        while True:
            dt = t0 + ta - time.perf_counter()
            if dt <= 0:
                break
            time.sleep(min(dt, 0.0005))
        idx, xs, vs = pre[q]
        e = engs[c]
        e.set_ti(ti)
        e.calc_firsthalf(len(clusters[c][0]), idx, xs, vs, EPS2)
        e.calc_lasthalf2()
        lat[q] = time.perf_counter() - (t0 + ta)
    wall = time.perf_counter() - t0
    for e in engs:
        e.close()
    inter = sum(ni * len(clusters[c][0]) for (_, c, ni, _, _) in calls)
    return lat, wall, inter
