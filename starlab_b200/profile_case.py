"""Run a few force calls of one shape through the C ABI (for profilers).

    python -m starlab_b200.profile_case --n 262144 --ni 16384 --mode mixed --calls 3

Loads an N-particle Plummer/Salpeter cluster into j-memory, then issues
`calls` g6calc_firsthalf_/g6calc_lasthalf2_ pairs of ni i-particles each at
new block times (so every call runs the predictor and the force kernel).
Prints the engine's device times.  Used to capture one force-kernel launch
under a profiler on a bounded case.
"""
import argparse
import json
import os

import numpy as np

from . import G6Engine, ics


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--ni", type=int, default=16384)
    ap.add_argument("--mode", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--eps2", type=float, default=1e-8)
    ap.add_argument("--h2", type=float, default=0.0)
    ap.add_argument("--config", default="", help="il,r,warps,h,nsplit")
    a = ap.parse_args()
    os.environ.setdefault("G6B200_EVENT_TIMING", "1")  # per-call device times in the stats
    m, x, v = ics.plummer(a.n, 11, masses=ics.salpeter_masses(a.n, 12))
    z = np.zeros((a.n, 3))
    eng = G6Engine(cluster_id=0, precision=a.mode, npipes=max(a.ni, 1))
    if a.config:
        eng.set_config(*[int(t) for t in a.config.split(",")])
    eng.set_j_particles(0.0, m, z, z, v, x)
    idx = np.arange(a.ni, dtype=np.int32)
    h2 = None if a.h2 <= 0 else np.full(a.ni, a.h2)
    for c in range(a.calls):
        eng.set_ti(1e-3 * (c + 1))
        eng.calc_firsthalf(a.n, idx, x[:a.ni], v[:a.ni], a.eps2, h2)
        eng.calc_lasthalf2()
        if h2 is not None:
            eng.read_neighbour_list()
        st = eng.stats()
        print(json.dumps(dict(call=c, force_ms=st["last_force_ms"], predict_ms=st["last_predict_ms"],
                              call_ms=st["last_call_ms"], config=eng.last_config(),
                              interactions_per_s=a.ni * a.n / (st["last_force_ms"] * 1e-3))))
    eng.close()


if __name__ == "__main__":
    main()
