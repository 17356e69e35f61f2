"""The multi-cluster ensemble integrator (batched, device-resident).

* forces at t = 0 of every cluster against the FP64 oracle;
* a cluster integrated alone and inside a mix of other clusters follows a
  bit-identical trajectory (its work items never depend on the others);
* block steps scheduled inside the predict kernel and the corrector (the
  steady state) and block steps through the schedule kernel give
  bit-identical states;
* the batched path and the plain one-call-per-cluster path agree, and both
  conserve energy (4th-order Hermite, eta = 0.02, t = 1/8).
"""
import numpy as np
import pytest

from helpers import rel_err, rel_err_vec

pytestmark = pytest.mark.gpu


def clusters(ns, seed):
    from starlab_b200 import ics
    out = []
    for k, n in enumerate(ns):
        m, x, v = ics.plummer(n, seed + k)
        out.append((m, x, v, (4.0 / n) ** 2))
    return out


def make(cl, precision="mixed"):
    from starlab_b200.ensemble import Ensemble
    return Ensemble([c[0] for c in cl], [c[1] for c in cl], [c[2] for c in cl], [c[3] for c in cl],
                    eta=0.02, precision=precision)


@pytest.mark.parametrize("precision,tol", [("mixed", (1e-6, 1e-5)), ("fp64", (1e-12, 1e-11))])
def test_start_forces_match_oracle(precision, tol, oracle):
    cl = clusters([300, 1000, 2048, 4100], 10)
    ens = make(cl, precision)
    ens.start()
    for c, (m, x, v, eps2) in enumerate(cl):
        st = ens.get(c)
        n = len(m)
        samp = np.arange(0, n, max(1, n // 200))
        ra, rj, rp, rn, _ = oracle.force(x, v, m, samp, x[samp], v[samp], eps2)
        assert rel_err_vec(st["acc"][samp], ra).max() <= tol[0]
        assert rel_err_vec(st["jerk"][samp], rj).max() <= tol[1]
        assert np.all(st["dt"] > 0) and np.all(st["dt"] <= 1.0 / 16)
    ens.close()


def test_alone_and_in_the_mix_are_bit_identical():
    cl = clusters([700, 1500, 256, 3000, 900], 30)
    mix = make(cl)
    alone = make([cl[3]])
    mix.start()
    alone.start()
    mix.run(1.0 / 32, tune=False)
    alone.run(1.0 / 32, tune=False)
    a = alone.get(0)
    b = mix.get(3)
    for k in ("x", "v", "acc", "jerk", "t", "dt"):
        assert np.array_equal(a[k], b[k]), k
    assert np.all(a["t"] == 1.0 / 32)
    mix.close()
    alone.close()


def test_fused_schedule_matches_the_schedule_kernel(monkeypatch):
    """Block steps whose members and block time come from the previous
    corrector and the predict kernel (atomic slot order) give bit-identical
    states to block steps through the schedule kernel (address order)."""
    cl = clusters([700, 1500, 256, 3000, 900], 31)
    out = []
    for fused in ("1", "0"):
        monkeypatch.setenv("G6B200_ENS_FUSED", fused)
        e = make(cl)
        e.start()
        st = e.run(1.0 / 32, tune=False)
        out.append((st, [e.get(c) for c in range(len(cl))]))
        e.close()
    (s1, a), (s0, b) = out
    assert s1["interactions"] == s0["interactions"] and s1["iterations"] == s0["iterations"]
    assert s1["launches"] < s0["launches"]
    for c in range(len(cl)):
        for k in ("x", "v", "acc", "jerk", "t", "dt"):
            assert np.array_equal(a[c][k], b[c][k]), (c, k)


def test_batched_and_per_cluster_agree_and_conserve_energy():
    cl = clusters([512, 1024, 2000], 50)
    e1, e2 = make(cl), make(cl)
    e1.start()
    e2.start()
    ek0, ep0 = e1.energies()
    s1 = e1.run(0.125, tune=True)
    s2 = e2.run(0.125, per_cluster=True)
    assert s1["interactions"] > 0 and s2["interactions"] > 0
    # same schedule: the same number of pair interactions to within the
    # few steps where rounding moved a timestep across a power of two
    assert abs(s1["interactions"] - s2["interactions"]) <= 0.05 * s2["interactions"]
    for ens in (e1, e2):
        ek, ep = ens.energies()
        de = np.abs((ek + ep) - (ek0 + ep0)) / np.abs(ek0 + ep0)
        assert de.max() < 1e-5, de
    for c in range(3):
        a, b = e1.get(c), e2.get(c)
        assert np.all(a["t"] == 0.125) and np.all(b["t"] == 0.125)
        assert np.max(np.abs(a["x"] - b["x"])) < 1e-4
    e1.close()
    e2.close()
