"""Generate the committed GRAPE-4 golden vectors from the reference itself.

Runs the reference's IEEE GRAPE-4 simulator (src/harpsims/harp3fastsim.c,
compiled as it is into oracle/_ref/libharp3sim.so by oracle/build_ref.py)
through its own ABI on small seeded inputs, and stores inputs and outputs
(acc, jerk, neighbour lists; the simulator returns no potential) as
g4_*.npz fixtures next to this script.  They pin the oracle's GRAPE-4
restatement (oracle/g4_oracle.c, tests/test_g4_oracle.py) where the
reference tree is absent, and the engine's GRAPE-4 ABI on the GPU.

The cases follow how kira drives the ABI (hdyn_grape4.C): the block's own
particles stored at the block time (so each i meets itself at r2 == 0),
eps2 == 0, per-slot neighbour spheres, padding with copies of the last i and
the slot pairs of a USE_HALF_CHIP build; plus softened and coincident-particle
cases.  All stay inside the simulator's static limits (1000 j, lists below
1024).

Usage: python tests/golden/make_golden_g4.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle.oracle import G4Oracle, Harp3Sim  # noqa: E402
from starlab_b200 import ics  # noqa: E402


def j_state(n, seed, salpeter=False):
    masses = ics.salpeter_masses(n, seed + 50) if salpeter else None
    m, x, v = ics.plummer(n, seed, masses=masses)
    rng = np.random.default_rng(seed + 7)
    aj = 0.5 * (-x / (1.0 + np.sum(x * x, axis=1, keepdims=True)) ** 1.5)
    jj = rng.normal(scale=0.5, size=(n, 3)) / 6.0
    t = rng.uniform(0.0, 0.01, n)
    return m, x, v, aj, jj, t


def kira_block(seed, n=600, nblock=40, half_chip=False, npipe=None):
    """Block members re-stored at ti = the block time (hdyn_grape4.C:1203-1222)."""
    m, x, v, aj, jj, t = j_state(n, seed)
    ti = 0.0125
    rng = np.random.default_rng(seed)
    block = np.sort(rng.choice(n, nblock, replace=False))
    xp, vp = G4Oracle().predict(ti, t, x, v, aj, jj)
    x, v, t = x.copy(), v.copy(), t.copy()
    x[block], v[block], t[block] = xp[block], vp[block], ti
    d2 = np.sum((x[block, None, :] - x[None, :, :]) ** 2, axis=2)
    d2[np.arange(nblock), block] = np.inf
    dnn = np.min(d2, axis=1)
    # kira's first guesses: about the nn distance, sometimes zero (no check)
    h2 = dnn * rng.uniform(0.5, 4.0, nblock)
    h2[rng.random(nblock) < 0.25] = 0.0
    xi, vi = x[block], v[block]
    eps2 = np.zeros(nblock)
    if half_chip:
        xi, vi, eps2, h2 = (np.repeat(a, 2, axis=0) for a in (xi, vi, eps2, h2))
    if npipe:
        pad = npipe - xi.shape[0]
        xi, vi, eps2, h2 = (np.concatenate([a, np.repeat(a[-1:], pad, axis=0)]) for a in (xi, vi, eps2, h2))
    return dict(m=m, x=x, v=v, aj=aj, jj=jj, t=t, ti=ti, xi=xi, vi=vi, eps2=eps2, h2=h2)


def softened(seed, n=997):
    m, x, v, aj, jj, t = j_state(n, seed, salpeter=True)
    rng = np.random.default_rng(seed)
    ni = 50
    xi = rng.normal(scale=0.6, size=(ni, 3))
    vi = rng.normal(scale=0.5, size=(ni, 3))
    eps2 = rng.choice([1e-4, 1e-6, 2.5e-5], ni)
    h2 = rng.choice([0.0, 0.003, 0.02, 0.08], ni)
    return dict(m=m, x=x, v=v, aj=aj, jj=jj, t=t, ti=0.02, xi=xi, vi=vi, eps2=eps2, h2=h2)


def coincident(seed, n=100):
    """Particles sharing positions exactly: every r2 == 0 pair is skipped
    when eps2 == 0, and counted (with its potential) when eps2 > 0."""
    m, x, v, aj, jj, t = j_state(n, seed)
    t[:] = 0.0
    x[10], x[11], x[12] = x[5], x[5], x[5]
    v[10] = v[5] + 0.1
    ti = 0.0
    xi = x[[5, 10, 20, 5]]
    vi = v[[5, 10, 20, 5]]
    eps2 = np.array([0.0, 0.0, 0.0, 1e-4])
    h2 = np.array([1e-3, 1e-3, 0.0, 1e-3])
    return dict(m=m, x=x, v=v, aj=aj, jj=jj, t=t, ti=ti, xi=xi, vi=vi, eps2=eps2, h2=h2)


CASES = {
    "g4_kira_block_n600": lambda: kira_block(11),
    "g4_kira_halfchip_padded_n600": lambda: kira_block(12, nblock=10, half_chip=True, npipe=32),
    "g4_softened_salpeter_n997": lambda: softened(13),
    "g4_coincident_n100": lambda: coincident(14),
}


def run_sim(sim, d):
    n = d["x"].shape[0]
    sim.load(d["x"], d["v"], d["aj"], d["jj"], d["m"], d["t"])
    acc, jerk, lists = sim.force(d["ti"], n, d["xi"], d["vi"], d["eps2"], d["h2"])
    off = np.zeros(len(lists) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(a) for a in lists])
    idx = np.concatenate(lists).astype(np.int32) if off[-1] else np.zeros(0, np.int32)
    return dict(acc=acc, jerk=jerk, nb_off=off, nb_idx=idx)


def main():
    sim = Harp3Sim()
    for name, make in CASES.items():
        d = make()
        d.update(run_sim(sim, d))
        d["ti"] = np.float64(d["ti"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print("wrote", name, "ni", d["xi"].shape[0], "nb", int(d["nb_off"][-1]))


if __name__ == "__main__":
    main()
