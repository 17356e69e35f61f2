"""The oracle's CPU GRAPE-6 ABI (oracle/g6_abi_oracle.c) under Starlab's
own tools (CPU only).

The reference has no GRAPE-6 emulator, so the CPU runs of its GRAPE-6
branch that the GPU library is compared with come from this file.  Here it
is pinned against the reference's CPU paths:

  * get_densities over it computes, for every particle whose sphere
    converged, exactly the density of the CPU tool compute_density -k 12;
  * kira over it (GRAPE-6 branch, kira_ev.C:886) starts at kira -0's energy
    and conserves energy as well (within 2x over t = 0.5).
"""
import os
import re
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref")


def _exes(*names):
    p = [os.path.join(REF, n) for n in names]
    if not all(os.path.exists(x) for x in p):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    return p


def _run(cmd, snap, cwd):
    with open(snap) as fin:
        r = subprocess.run(cmd, stdin=fin, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=300,
                           cwd=cwd)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout, r.stderr


def _snap(tmp_path, mk, n, seed):
    p = tmp_path / ("p%d.snap" % n)
    with open(p, "w") as f:
        subprocess.run([mk, "-n", str(n), "-s", str(seed), "-i"], stdout=f, stderr=subprocess.DEVNULL, check=True)
    return p


def test_get_densities_over_the_oracle_matches_compute_density(tmp_path):
    mk, gd, cd = _exes("makeplummer", "get_densities_g6o", "compute_density")
    snap = _snap(tmp_path, mk, 3000, 8)
    out_o, err_o = _run([gd, "-v"], snap, tmp_path)
    out_c, _ = _run([cd, "-k", "12"], snap, tmp_path)
    assert "GPU acceleration" in err_o

    def dens(out):
        return np.array([float(m.group(1)) for m in re.finditer(r"^\s+density\s+=\s+(\S+)\s*$", out, re.M)])

    do, dc = dens(out_o), dens(out_c)
    assert do.size == dc.size == 3000
    ok = do > 0
    assert ok.sum() > 1500
    assert np.array_equal(do[ok], dc[ok])


def test_kira_grape6_branch_on_the_oracle(tmp_path):
    mk, kira, kg6o = _exes("makeplummer", "kira", "kira_g6o")
    snap = _snap(tmp_path, mk, 512, 42)
    args = ["-t", "0.5", "-d", "0.125", "-e", "0.001", "-a", "0.02"]

    def energies(cmd):
        _, err = _run(cmd, snap, tmp_path)
        return err, [float(m.group(1)) for m in re.finditer(r"Energies:\s+\S+\s+\S+\s+(\S+)", err)]

    log, eo = energies([kg6o] + args)
    _, ec = energies([kira, "-0"] + args)
    assert "GPU acceleration" in log
    assert len(eo) >= 4 and eo[0] == pytest.approx(ec[0], rel=1e-12)
    deo = max(abs(e - eo[0]) for e in eo[1:])
    dec = max(abs(e - ec[0]) for e in ec[1:])
    assert deo <= 2.0 * dec, (deo, dec)
