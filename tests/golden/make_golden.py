"""Generate the committed golden vectors from the reference itself.

Runs Starlab's own FP64 force path (oracle/_ref/libref_force.so: the
reference's predict_loworder + hdyn::flat_calculate_acc_and_jerk, compiled
from its sources by oracle/build_ref.py) on small seeded inputs and stores
inputs and outputs as .npz fixtures next to this script.  The fixtures pin
the oracle's C restatement (tests/test_oracle.py) on machines where the
reference tree is absent.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle.oracle import RefForce  # noqa: E402
from starlab_b200 import ics  # noqa: E402

CASES = [
    # name, n, seed, eps, dt-scale, salpeter
    ("plummer_n64_eps1e-3", 64, 1, 1e-3, 0.01, False),
    ("plummer_n300_eps1e-2", 300, 2, 1e-2, 0.02, False),
    ("salpeter_n257_eps1e-4", 257, 3, 1e-4, 0.005, True),
    ("plummer_n128_eps0", 128, 4, 0.0, 0.001, False),
]


def make(ref, n, seed, eps, dts, salpeter):
    masses = ics.salpeter_masses(n, seed + 50) if salpeter else None
    m, x, v = ics.plummer(n, seed, masses=masses)
    rng = np.random.default_rng(seed + 99)
    a = rng.normal(size=(n, 3))
    j = rng.normal(size=(n, 3))
    tj = rng.uniform(0.0, dts, n)
    ti = dts
    out = ref.force(m, x, v, a, j, tj, ti, eps, want_pred=True)
    return dict(mass=m, pos=x, vel=v, acc_in=a, jerk_in=j, tj=tj, ti=np.float64(ti), eps=np.float64(eps),
                eps2=np.float64(out["eps2"]), pred_pos=out["pred_pos"], pred_vel=out["pred_vel"],
                acc=out["acc"], jerk=out["jerk"], pot=out["pot"], nn=out["nn"], dnn_sq=out["dnn_sq"])


def main():
    ref = RefForce()
    for name, n, seed, eps, dts, salp in CASES:
        d = make(ref, n, seed, eps, dts, salp)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print("wrote", name)


if __name__ == "__main__":
    main()
