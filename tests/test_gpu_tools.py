"""Starlab's own tools driving the GRAPE-6 engine through the unchanged ABI.

hsys_stats, hscale and get_densities call the GRAPE when one is configured
(grape6_calculate_energies, hdyn_grape6.C:1403-1546;
grape6_calculate_densities, :4283-4450).  oracle/build_ref.py links them
against libg6b200.so ahead of the null stubs (*_g6), and the same mains
against the oracle's CPU GRAPE-6 (*_g6o, oracle/g6_abi_oracle.c); the CPU
runs are the oracle:

  * hsys_stats_g6 energies == hsys_stats (CPU) energies (FP64: 1e-12;
    mixed: 1e-6);
  * hscale_g6 output == hscale output (positions and velocities, 1e-12);
  * get_densities_g6 densities == get_densities_g6o densities, particle by
    particle, zeros included: the GRAPE path adjusts each neighbour sphere
    until it holds 12 others (hdyn_grape6.C:3704-3893) and gives up with
    density 0 after 20 force passes or beyond h2_crit (:4079-4282), so the
    same lists must lead to the same decisions; and every density it does
    compute equals the reference's CPU tool compute_density -k 12, which
    the GRAPE path feeds the 12-neighbour candidates.

The GRAPE-4 branch of get_densities dereferences a null kira_options
pointer right after opening the GRAPE (hdyn_grape4.C:1994, where the GRAPE-6
version checks it, hdyn_grape6.C:173), so it is not run.
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref")


def _need(name):
    p = os.path.join(REF, name)
    if not os.path.exists(p):
        pytest.skip("%s not built (python oracle/build_ref.py on a machine with the reference)" % name)
    return p


def _run(exe, args, snap, cwd, env=None):
    e = dict(os.environ)
    e.update(env or {})
    with open(snap) as fin:
        r = subprocess.run([exe] + args, stdin=fin, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                           timeout=600, cwd=cwd, text=True, env=e)
    assert r.returncode == 0, r.stderr[-3000:]
    return r.stdout, r.stderr


def _energies(log):
    return [tuple(float(x) for x in m.groups()) for m in re.finditer(r"Energies:\s+(\S+)\s+(\S+)\s+(\S+)", log)]


def _vectors(out, key):
    return np.array([[float(x) for x in m.groups()]
                     for m in re.finditer(r"^\s+%s\s+=\s+(\S+)\s+(\S+)\s+(\S+)\s*$" % key, out, re.M)])


@pytest.fixture(scope="module")
def snaps(tmp_path_factory):
    mk = _need("makeplummer")
    d = tmp_path_factory.mktemp("tools")
    out = {}
    for n, seed in ((1024, 42), (4000, 3)):
        p = os.path.join(d, "p%d.snap" % n)
        with open(p, "w") as f:
            subprocess.run([mk, "-n", str(n), "-s", str(seed), "-i"], stdout=f, stderr=subprocess.DEVNULL, check=True)
        out[n] = p
    return str(d), out


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_hsys_stats_energies(snaps, precision, tol):
    d, s = snaps
    _, cpu = _run(_need("hsys_stats"), [], s[1024], d)
    _, g6 = _run(_need("hsys_stats_g6"), [], s[1024], d, {"G6B200_PRECISION": precision})
    assert "GPU acceleration" in g6
    ec, eg = _energies(cpu), _energies(g6)
    assert ec and eg
    assert np.allclose(eg[0], ec[0], rtol=tol, atol=0), (eg[0], ec[0])


def test_hscale_rescales_like_the_cpu_tool(snaps):
    d, s = snaps
    args = ["-e", "-0.5", "-q", "0.4", "-m", "1"]
    out_c, _ = _run(_need("hscale"), args, s[1024], d)
    out_g, err_g = _run(_need("hscale_g6"), args, s[1024], d, {"G6B200_PRECISION": "fp64"})
    assert "GPU acceleration" in err_g
    for key in ("r", "v"):
        a, b = _vectors(out_g, key), _vectors(out_c, key)
        assert a.shape == b.shape and a.shape[0] >= 1024
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), key


def _densities(out):
    return np.array([float(m.group(1)) for m in re.finditer(r"^\s+density\s+=\s+(\S+)\s*$", out, re.M)])


def test_get_densities_matches_its_cpu_runs(snaps):
    d, s = snaps
    out_o, _ = _run(_need("get_densities_g6o"), ["-v"], s[4000], d)
    out_c, _ = _run(_need("compute_density"), ["-k", "12"], s[4000], d)
    out_g, err_g = _run(_need("get_densities_g6"), ["-v"], s[4000], d, {"G6B200_PRECISION": "fp64"})
    assert "GPU acceleration" in err_g
    do, dc, dg = _densities(out_o), _densities(out_c), _densities(out_g)
    assert do.size == dc.size == dg.size == 4000, (do.size, dc.size, dg.size)
    assert np.array_equal(dg, do), np.flatnonzero(dg != do)[:10]
    ok = dg > 0
    assert ok.sum() > 0.5 * dg.size
    assert np.array_equal(dg[ok], dc[ok])
