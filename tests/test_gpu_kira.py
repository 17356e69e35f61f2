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


def _trace(log, key):
    m = re.search(r"g6b200\[0\] trace: .*?%s (\d+)" % key, log)
    return int(m.group(1)) if m else None


@pytest.fixture(scope="module")
def binaries1024(tmp_path_factory):
    """N = 1024 Plummer sphere (seed 42) with primordial binaries from the
    reference's own generators: makesecondary gives 10% of the stars a
    secondary (mass ratio >= 0.25), makebinary puts them on orbits of
    0.5-2 kT (soft enough that some binaries' perturber lists overflow)."""
    tools = [_need(t) for t in ("makeplummer", "makesecondary", "makebinary")]
    d = tmp_path_factory.mktemp("kira_bin")
    snap = os.path.join(d, "b1024.snap")
    p1 = subprocess.Popen([tools[0], "-n", "1024", "-s", "42", "-i"], stdout=subprocess.PIPE,
                          stderr=subprocess.DEVNULL)
    p2 = subprocess.Popen([tools[1], "-f", "0.1", "-q", "-l", "0.25", "-s", "7"], stdin=p1.stdout,
                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL)
    with open(snap, "w") as f:
        p3 = subprocess.run([tools[2], "-f", "3", "-o", "3", "-l", "0.5", "-u", "2", "-s", "9"], stdin=p2.stdout,
                            stdout=f, stderr=subprocess.DEVNULL)
    p1.wait(), p2.wait()
    assert p3.returncode == 0
    return str(d), snap


BIN_ARGS = ["-t", "0.125", "-d", "0.0625", "-e", "0.001", "-a", "0.02"]


def test_kira_binaries_and_perturbation_calls(binaries1024):
    """kira's GRAPE-6 branch with binaries: the perturbation call
    (grape6_calculate_perturbation, hdyn_grape6.C:3415-3587, issued from
    hdyn_ev.C:3127 when a binary's perturber list overflows) sends ni = 2
    calls with both components under one index; the engine's trace counts
    them.  Energy error within 2x of the same kira branch over the CPU
    GRAPE-6 oracle (kira_g6o, oracle/g6_abi_oracle.c), which counts the
    same call shape; kira -0 (no GRAPE) is reported beside them."""
    d, snap = binaries1024
    gpu = run_kira(_need("kira_g6"), snap, BIN_ARGS, {"G6B200_PRECISION": "fp64", "G6B200_TRACE": "1"}, d)
    cpu_g6 = run_kira(_need("kira_g6o"), snap, BIN_ARGS, {"G6O_TRACE": "1"}, d)
    cpu = run_kira(_need("kira"), snap, ["-0"] + BIN_ARGS, {}, d)
    pairs = _trace(gpu, "pair_calls")
    m = re.search(r"g6 oracle trace: calls (\d+) pair_calls (\d+)", cpu_g6)
    assert pairs is not None and m is not None
    assert pairs > 0 and int(m.group(2)) > 0, (pairs, m.group(0))
    eg, eo, ec = energies(gpu), energies(cpu_g6), energies(cpu)
    assert eg[0] == pytest.approx(eo[0], rel=1e-12) and eg[0] == pytest.approx(ec[0], rel=1e-12)
    de_g = max(abs(e - eg[0]) for e in eg[1:])
    de_o = max(abs(e - eo[0]) for e in eo[1:])
    de_c = max(abs(e - ec[0]) for e in ec[1:])
    print("binaries: |dE| kira_g6 %.3e kira_g6o %.3e kira -0 %.3e; pair calls %d (oracle %s)"
          % (de_g, de_o, de_c, pairs, m.group(2)))
    assert de_g <= 2.0 * de_o, (de_g, de_o, de_c)


def test_kira_jp_buffer_mode_identical(plummer1024):
    """kira -2 batches j-particle writes through g6_initialize_jp_buffer_ /
    g6_flush_jp_buffer_ (hdyn_grape6.C:266-271, :672-673).  The engine
    stages j updates either way, so the run gives the same energies at every
    log point as the run without -2."""
    d, snap = plummer1024
    args = ["-t", "0.25", "-d", "0.0625", "-e", "0.001", "-a", "0.02"]
    plain = run_kira(_need("kira_g6"), snap, args, {"G6B200_PRECISION": "fp64"}, d)
    dma = run_kira(_need("kira_g6"), snap, ["-2"] + args, {"G6B200_PRECISION": "fp64"}, d)
    assert "g6_initialize_jp_buffer_" in dma
    ep, ed = energies(plain), energies(dma)
    assert len(ep) >= 4 and ep == ed, (ep, ed)



def test_kira_mixed_step_count_near_fp64(tmp_path):
    """kira in the mixed mode takes the FP64 run's steps, near enough: N =
    32768 Plummer (seed 42), calls of up to 4096 i (G6B200_NPIPES) so the
    large blocks run in mixed precision while blocks below 2^25
    interactions run in FP64, t = 1/32.  The force-call count stays within
    1.2x of the FP64 run's (with every call mixed it was 25x at N = 8192),
    and the mixed run did use the mixed kernels (particles refined)."""
    mk = _need("makeplummer")
    snap = os.path.join(tmp_path, "p32k.snap")
    with open(snap, "w") as f:
        subprocess.run([mk, "-n", "32768", "-s", "42", "-i"], stdout=f, stderr=subprocess.DEVNULL, check=True)
    args = ["-t", "0.03125", "-d", "0.015625", "-e", "0.001", "-a", "0.02"]
    runs = {}
    for prec in ("fp64", "mixed"):
        log = run_kira(_need("kira_g6"), snap, args,
                       {"G6B200_PRECISION": prec, "G6B200_NPIPES": "4096", "G6B200_TRACE": "1"}, str(tmp_path))
        runs[prec] = (_trace(log, "calls"), _trace(log, "refined"), energies(log))
    (c64, _, e64), (cmx, refined, emx) = runs["fp64"], runs["mixed"]
    print("kira N=32768: calls fp64 %d mixed %d, refined %d, dE fp64 %.2e mixed %.2e"
          % (c64, cmx, refined, abs(e64[-1] - e64[0]), abs(emx[-1] - emx[0])))
    assert cmx <= 1.2 * c64, (cmx, c64)
    assert refined > 0
    assert abs(emx[-1] - emx[0]) <= 1e-8 * abs(emx[0])
