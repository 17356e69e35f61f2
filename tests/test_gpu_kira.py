"""kira end to end: the unchanged reference integrator driving the engine.

oracle/_ref/kira_g6 is Starlab's own kira main linked against
libg6b200.so ahead of the reference's GRAPE stubs (the link order of
src/node/dyn/hdyn/evolve/Makefile.am:36-48), so g6_npipes_() > 0 and kira
takes its GRAPE-6 branch (kira_config.C:62; kira_ev.C:886).  The CPU run
(`kira -0`) of the same binary set is the oracle: an equal-mass Plummer
sphere of N = 1024 (reference makeplummer, seed 42), eps = 1e-3, eta = 0.02,
integrated to t = 1.  The GPU run in FP64 mode must keep the total-energy
error within 2x of the CPU run's (largest |de| over the log points).
"""
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref")

pytestmark = pytest.mark.gpu


def _need(name):
    p = os.path.join(REF, name)
    if not os.path.exists(p):
        pytest.skip("%s not built (python oracle/build_ref.py on a machine with the reference)" % name)
    return p


def run_kira(exe, snap, args, env_extra, tmp):
    env = dict(os.environ)
    env.update(env_extra)
    with open(snap) as fin:
        r = subprocess.run([exe] + args, stdin=fin, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                           env=env, timeout=600, cwd=tmp, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return r.stderr


def energies(log):
    tot = [float(m.group(1)) for m in re.finditer(r"Energies:\s+\S+\s+\S+\s+(\S+)", log)]
    return tot


@pytest.fixture(scope="module")
def plummer1024(tmp_path_factory):
    mk = _need("makeplummer")
    d = tmp_path_factory.mktemp("kira")
    snap = os.path.join(d, "p1024.snap")
    with open(snap, "w") as f:
        subprocess.run([mk, "-n", "1024", "-s", "42", "-i"], stdout=f, stderr=subprocess.DEVNULL, check=True)
    return str(d), snap


ARGS = ["-t", "1", "-d", "0.25", "-e", "0.001", "-a", "0.02"]


def test_kira_fp64_energy_within_2x_of_cpu(plummer1024):
    d, snap = plummer1024
    kira = _need("kira")
    kira_g6 = _need("kira_g6")
    cpu = run_kira(kira, snap, ["-0"] + ARGS, {}, d)
    gpu = run_kira(kira_g6, snap, ARGS, {"G6B200_PRECISION": "fp64"}, d)
    assert "GPU acceleration" in gpu or "GRAPE-6" in gpu, gpu[:2000]
    ec, eg = energies(cpu), energies(gpu)
    assert len(ec) >= 5 and len(eg) >= 5
    de_cpu = max(abs(e - ec[0]) for e in ec[1:])
    de_gpu = max(abs(e - eg[0]) for e in eg[1:])
    assert ec[0] == pytest.approx(eg[0], rel=1e-12)
    assert de_gpu <= 2.0 * de_cpu, (de_gpu, de_cpu)


def test_kira_mixed_runs_and_conserves(plummer1024):
    d, snap = plummer1024
    kira_g6 = _need("kira_g6")
    gpu = run_kira(kira_g6, snap, ARGS, {"G6B200_PRECISION": "mixed"}, d)
    eg = energies(gpu)
    de = max(abs(e - eg[0]) for e in eg[1:])
    assert de < 1e-6, de


def test_kira_recovers_from_injected_engine_error(plummer1024):
    """lasthalf2 fails once (host-side injection): kira resets, reopens,
    reloads j-memory and retries (hdyn_grape6.C:892-899), then finishes."""
    d, snap = plummer1024
    kira_g6 = _need("kira_g6")
    gpu = run_kira(kira_g6, snap, ["-t", "0.125", "-d", "0.125", "-e", "0.001", "-a", "0.02"],
                   {"G6B200_PRECISION": "fp64", "G6B200_FAULT_LASTHALF": "50"}, d)
    assert "Resetting GRAPE and retrying" in gpu
    assert len(energies(gpu)) >= 2
