"""Pin the GRAPE-4 oracle against the reference's GRAPE-4 simulator (CPU only).

1. Golden vectors (tests/golden/g4_*.npz) made by
   tests/golden/make_golden_g4.py with the reference's own simulator
   (src/harpsims/harp3fastsim.c): from the same inputs the restatement
   (oracle/g4_oracle.c) must reproduce acc, jerk and every neighbour list
   bit for bit (same predictor and pair loop, same j order).
2. When oracle/_ref is built here, the same on fresh seeded inputs.
3. The potential, which the simulator leaves at 0, is checked against the
   GRAPE-6 oracle's (the reference pair formula, hdyn_ev.C:2019-2036) where
   both define it.
4. libh3b200.so loads without a GPU and exports every entry point
   include/h3b200.h declares; libg6b200.so exports none of them (kira picks
   the GRAPE-4 branch whenever h3npipe_() answers, kira_config.C:65-95).
"""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "g4_*.npz")))
HEADER = os.path.join(REPO, "include", "h3b200.h")


@pytest.fixture(scope="module")
def g4o():
    from oracle.oracle import G4Oracle
    return G4Oracle()


def lists_of(g):
    off, idx = g["nb_off"], g["nb_idx"]
    return [idx[off[i]:off[i + 1]] for i in range(len(off) - 1)]


def test_g4_golden_fixtures_present():
    assert len(GOLDEN) >= 4


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_g4_oracle_matches_simulator_golden(path, g4o):
    g = np.load(path)
    xp, vp = g4o.predict(float(g["ti"]), g["t"], g["x"], g["v"], g["aj"], g["jj"])
    acc, jerk, pot, cnt, nb = g4o.force(xp, vp, g["m"], g["xi"], g["vi"], g["eps2"], g["h2"])
    assert np.array_equal(acc, g["acc"])
    assert np.array_equal(jerk, g["jerk"])
    want = lists_of(g)
    assert all(np.array_equal(a, b) for a, b in zip(nb, want))
    assert np.all(pot < 0)


def test_g4_kira_block_meets_itself_at_zero_distance(g4o):
    """eps2 == 0 and the block stored at the block time: the i's own
    j-record sits at r2 == 0, so it is skipped by the force and listed as
    its own neighbour whenever h2 > 0 (kira's get_neighbors_and_adjust_h2
    needs >= 2 entries, hdyn_grape4.C:881)."""
    g = np.load(os.path.join(HERE, "golden", "g4_kira_block_n600.npz"))
    xp, _ = g4o.predict(float(g["ti"]), g["t"], g["x"], g["v"], g["aj"], g["jj"])
    for k, lst in enumerate(lists_of(g)):
        self_j = np.flatnonzero(np.all(xp == g["xi"][k], axis=1))
        assert self_j.size == 1
        assert (self_j[0] in lst) == (g["h2"][k] > 0)


def test_g4_coincident_pairs(g4o):
    g = np.load(os.path.join(HERE, "golden", "g4_coincident_n100.npz"))
    lists = lists_of(g)
    # slot 0 and slot 3 share the position of j = 5, 10, 11, 12; eps2 = 0 skips all
    # four in the force but lists them; eps2 > 0 counts them.
    assert set([5, 10, 11, 12]) <= set(lists[0].tolist())
    assert np.all(np.isfinite(g["acc"])) and np.all(np.isfinite(g["jerk"]))
    _, _, pot, _, _ = g4o.force(g["x"], g["v"], g["m"], g["xi"], g["vi"], g["eps2"], g["h2"])
    m = g["m"]
    # the softened slot sees the four coincident masses at r = sqrt(2 eps2)
    extra = (m[5] + m[10] + m[11] + m[12]) / np.sqrt(2 * g["eps2"][3])
    assert pot[3] < pot[0] - 0.99 * extra


def _sim_or_skip():
    from oracle.oracle import HARP3_LIB, Harp3Sim
    if not os.path.exists(HARP3_LIB):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    return Harp3Sim()


@pytest.mark.parametrize("n,seed,eps2", [(1000, 21, 0.0), (333, 22, 1e-4), (64, 23, 1e-2)])
def test_g4_oracle_matches_simulator_fresh(n, seed, eps2, g4o):
    from starlab_b200 import ics
    sim = _sim_or_skip()
    m, x, v = ics.plummer(n, seed)
    rng = np.random.default_rng(seed)
    aj, jj = rng.normal(size=(n, 3)) * 0.3, rng.normal(size=(n, 3)) * 0.1
    t = rng.uniform(0, 0.02, n)
    ti = 0.03
    sim.load(x, v, aj, jj, m, t)
    ni = 17
    xi = rng.normal(scale=0.5, size=(ni, 3))
    vi = rng.normal(scale=0.5, size=(ni, 3))
    h2 = rng.choice([0.0, 0.01, 0.05], ni)
    acc, jerk, lists = sim.force(ti, n, xi, vi, eps2, h2)
    xp, vp = g4o.predict(ti, t, x, v, aj, jj)
    oa, oj, op, cnt, nb = g4o.force(xp, vp, m, xi, vi, eps2, h2)
    assert np.array_equal(acc, oa) and np.array_equal(jerk, oj)
    assert all(np.array_equal(a, b) for a, b in zip(lists, nb))


def test_g4_potential_matches_the_reference_pair_formula(g4o, oracle):
    """Distinct positions, eps2 = 0: the GRAPE-4 pot equals the GRAPE-6
    oracle's (index exclusion) to rounding."""
    from starlab_b200 import ics
    m, x, v = ics.plummer(300, 31)
    idx = np.arange(0, 300, 7)
    _, _, pot4, _, _ = g4o.force(x, v, m, x[idx], v[idx], 0.0, 0.0)
    _, _, pot6, _, _ = oracle.force(x, v, m, idx, x[idx], v[idx], 0.0)
    assert np.max(np.abs(pot4 - pot6) / np.abs(pot6)) < 1e-13


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:unsigned\s+)?[a-z_0-9]+\s*\*?\s*([a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_h3_header_declares_the_reference_abi():
    names = declared_functions()
    ref = ["h3open_", "h3close_", "h3npipe_", "h3setnboards_", "h3getnboards_", "h3wait_", "h3setti_",
           "h3setmode_", "h3setled_", "h3jpmax_", "h3jpdma_indirect_", "h3mjpdma_indirect_", "h3mjpdma_start_",
           "h3mjpdma_flush_", "h3calc_", "h3calc_firsthalf_", "h3calc_lasthalf_", "h3nbread_", "h3nblist_",
           "count_nblist_low", "h3setdebuglevel_", "h3checkdmabuffers_", "set_time_check_mode"]
    assert not [r for r in ref if r not in names]


def test_h3_library_exports_every_declared_symbol():
    from starlab_b200.grape4 import LIB_PATH
    from starlab_b200 import LIB_PATH as G6_LIB
    lib = ctypes.CDLL(LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", G6_LIB], stdout=subprocess.PIPE, text=True).stdout
    g6_exports = set(l.split()[-1] for l in out.splitlines())
    assert not [n for n in declared_functions() if n in g6_exports and not n.startswith("g6")]


def test_h3_npipe_without_device():
    import sys
    from starlab_b200.grape4 import LIB_PATH
    code = "import ctypes,sys; lib=ctypes.CDLL(sys.argv[1]); print(lib.h3npipe_(), lib.h3jpmax_(), lib.h3getnboards_())"
    env = dict(os.environ, H3B200_NPIPES="96")
    r = subprocess.run([sys.executable, "-c", code, LIB_PATH], env=env, stdout=subprocess.PIPE, text=True)
    assert r.stdout.split() == ["96", "1048576", "1"]


def test_kira_grape4_branch_on_the_oracle_pipeline(tmp_path):
    """Starlab's kira, GRAPE-4 branch, over the oracle's CPU pipeline
    (oracle/h3_oracle.c): the integration the GPU library is compared
    with.  The branch computes without softening (hdyn_grape4.C:320-330), so
    the initial energy is the unsoftened Plummer value, -1/4; its energy
    error over t = 0.5 stays within 2x of kira -0's."""
    import re
    ref = os.path.join(REPO, "oracle", "_ref")
    exes = [os.path.join(ref, n) for n in ("makeplummer", "kira", "kira_g4o")]
    if not all(os.path.exists(e) for e in exes):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    snap = tmp_path / "p.snap"
    with open(snap, "w") as f:
        subprocess.run([exes[0], "-n", "512", "-s", "42", "-i"], stdout=f, stderr=subprocess.DEVNULL, check=True)
    args = ["-t", "0.5", "-d", "0.125", "-e", "0.001", "-a", "0.02"]

    def energies(cmd):
        with open(snap) as fin:
            r = subprocess.run(cmd, stdin=fin, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True,
                               timeout=300, cwd=tmp_path)
        assert r.returncode == 0, r.stderr[-2000:]
        return r.stderr, [float(m.group(1)) for m in re.finditer(r"Energies:\s+\S+\s+\S+\s+(\S+)", r.stderr)]

    log, e4 = energies([exes[2]] + args)
    _, e0 = energies([exes[1], "-0"] + args)
    assert "found GRAPE-4 acceleration" in log
    assert len(e4) >= 4 and e4[0] == pytest.approx(-0.25, abs=1e-14)
    de4 = max(abs(e - e4[0]) for e in e4[1:])
    de0 = max(abs(e - e0[0]) for e in e0[1:])
    assert de4 <= 2.0 * de0, (de4, de0)
