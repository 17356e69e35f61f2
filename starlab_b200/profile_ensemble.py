"""Run one slice of the batched ensemble workload (for profilers).

    python -m starlab_b200.profile_ensemble --t 0.015625

The bench's ensemble: 256 equal-mass Plummer clusters, N log-uniform in
[256, 16384] (seed 2024), eps^2 = (4/N)^2, eta = 0.02, mixed precision;
started at t = 0 and advanced to --t (no tuning unless --tune).  Prints the
run's statistics as one JSON line.
"""
import argparse
import json

import numpy as np

from . import ics
from .ensemble import Ensemble


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clusters", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--t", type=float, default=1.0 / 64)
    ap.add_argument("--tune", action="store_true")
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    ns = np.exp(rng.uniform(np.log(256), np.log(16384), a.clusters)).astype(int)
    cl = [ics.plummer(int(n), a.seed * 1000 + k) for k, n in enumerate(ns)]
    e = Ensemble([c[0] for c in cl], [c[1] for c in cl], [c[2] for c in cl], (4.0 / ns) ** 2, eta=0.02,
                 precision="mixed")
    e.start()
    st = e.run(a.t, tune=a.tune)
    st["interactions_per_s"] = st["interactions"] / st["seconds"]
    st["us_per_iteration"] = st["seconds"] / st["iterations"] * 1e6
    print(json.dumps(st))


if __name__ == "__main__":
    main()
