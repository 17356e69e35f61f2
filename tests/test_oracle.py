"""Pin the oracle's C restatement against the reference (CPU only).

1. Golden vectors (tests/golden/*.npz) made by tests/golden/make_golden.py
   from Starlab's own FP64 path: given the reference's predicted positions,
   the restated force loop must reproduce acc, jerk, pot, nn and d_nn_sq
   bit for bit (same pair formula and j order, hdyn_ev.C:2019-2036,
   2128-2222); the restated predictor (a/2, j/6 form) must agree to within
   a few ulps.
2. When oracle/_ref is built here, the same comparison on fresh seeded
   inputs, including the threaded reference driver.
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(p for p in glob.glob(os.path.join(HERE, "golden", "*.npz"))
                if not os.path.basename(p).startswith(("g4_", "story_")))


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 4


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path, oracle):
    g = np.load(path)
    n = g["mass"].shape[0]
    acc, jerk, pot, nn, nn_r2 = oracle.force(g["pred_pos"], g["pred_vel"], g["mass"], np.arange(n),
                                             g["pred_pos"], g["pred_vel"], float(g["eps2"]))
    assert np.array_equal(acc, g["acc"])
    assert np.array_equal(jerk, g["jerk"])
    assert np.array_equal(pot, g["pot"])
    assert np.array_equal(nn, g["nn"])
    assert np.array_equal(nn_r2, g["dnn_sq"])
    xp, vp = oracle.predict(float(g["ti"]), g["tj"], g["pos"], g["vel"], 0.5 * g["acc_in"], g["jerk_in"] / 6.0)
    scale_x = np.abs(g["pred_pos"]).max()
    scale_v = np.abs(g["pred_vel"]).max()
    assert np.max(np.abs(xp - g["pred_pos"])) <= 4e-16 * scale_x
    assert np.max(np.abs(vp - g["pred_vel"])) <= 4e-16 * scale_v


def test_golden_eps0_case_has_no_softening():
    g = np.load(os.path.join(HERE, "golden", "plummer_n128_eps0.npz"))
    assert float(g["eps2"]) == 0.0
    assert np.all(g["pot"] < 0)


def _ref_or_skip():
    from oracle.oracle import REF_LIB, RefForce
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    return RefForce()


@pytest.mark.parametrize("n,eps,nthreads", [(200, 1e-3, 1), (1031, 1e-2, 1), (777, 3e-4, 4)])
def test_oracle_matches_reference_fresh(n, eps, nthreads, oracle):
    from starlab_b200 import ics
    ref = _ref_or_skip()
    m, x, v = ics.plummer(n, n)
    rng = np.random.default_rng(n)
    a, j = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    tj = rng.uniform(0, 0.01, n)
    out = ref.force(m, x, v, a, j, tj, 0.01, eps, nthreads=nthreads, want_pred=True)
    acc, jerk, pot, nn, nn_r2 = oracle.force(out["pred_pos"], out["pred_vel"], m, np.arange(n),
                                             out["pred_pos"], out["pred_vel"], out["eps2"])
    assert np.array_equal(acc, out["acc"]) and np.array_equal(jerk, out["jerk"])
    assert np.array_equal(pot, out["pot"]) and np.array_equal(nn, out["nn"])
    assert np.array_equal(nn_r2, out["dnn_sq"])


def test_oracle_neighbour_lists_brute_force(oracle):
    """Neighbour lists: ascending addresses, r^2 < h2 without softening,
    self included iff include_self (the npipes > 48 convention)."""
    from starlab_b200 import ics
    n = 600
    m, x, v = ics.plummer(n, 5)
    idx = np.arange(0, n, 7)
    h2 = 0.3 ** 2
    for inc in (True, False):
        lists = oracle.neighbours(x, idx, x[idx], h2, include_self=inc)
        for k, i in enumerate(idx):
            d2 = np.sum((x - x[i]) ** 2, axis=1)
            want = np.nonzero(d2 < h2)[0]
            if not inc:
                want = want[want != i]
            assert np.array_equal(lists[k], want)


def test_oracle_skips_self_by_index_not_address(oracle):
    from starlab_b200 import ics
    n = 50
    m, x, v = ics.plummer(n, 8)
    ids = np.arange(n) + 1000
    acc1, _, pot1, _, _ = oracle.force(x, v, m, ids[:5], x[:5], v[:5], 1e-4, jindex=ids)
    acc2, _, pot2, _, _ = oracle.force(x, v, m, np.arange(5), x[:5], v[:5], 1e-4)
    assert np.array_equal(acc1, acc2) and np.array_equal(pot1, pot2)
