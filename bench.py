#!/usr/bin/env python3
"""Benchmark of the B200 GRAPE-6 force engine.

Workload (one "step"): a full force sweep of an N = 262144 Plummer sphere
with a Salpeter mass spectrum (slope -2.35, 0.1-100, total mass 1),
eps^2 = 1e-8, in the engine's mixed-precision mode: predict all j to the
step's block time, then acc + jerk + pot + nearest neighbour on every
particle from every other one, 262144 x 262143 = 6.87e10 pair interactions.
Inputs are seeded synthetic stand-ins for the reference generators
(makeplummer | makemass); acc/jerk for the predictor come from one engine
sweep at t = 0.

Reported (one JSON line on rank 0):
  value        interactions/s with the j-set resident in HBM, timed on the
               device with CUDA events on the engine's stream (predictor +
               i-record build + force + split reduction), L2 flushed (256 MiB
               write) before every timed step; whole job over all ranks
  e2e          the same metric through the g6 C ABI with host buffers:
               every step uploads all j-particles (g6b200_set_j_particles),
               runs g6calc_firsthalf_/g6calc_lasthalf2_ over all i in npipes
               chunks from pinned staging, and reads results back
  roofline     force kernel vs the FP32 pipe: 60 flops per interaction (the
               acc+jerk convention) / mean force-kernel duration, against
               SMs x 128 FP32 lanes x 2 x max SM clock
  cpu_baseline Starlab's own FP64 force loop (oracle/_ref/libref_force.so,
               hdyn::flat_calculate_acc_and_jerk) on the host cores, on a
               bounded sample of i
  latency      p50/p99 of single force calls through the C ABI, ni drawn
               from a power law (slope -1) on [1, N]
  grape4       the GRAPE-4 ABI (libh3b200.so, FP64): a full sweep of an
               N = 65536 Plummer sphere through h3calc_ in h3npipe_() chunks,
               the block stored at the block time as kira's GRAPE-4 branch
               does; wall-clock interactions/s through the ABI
  story        story-format snapshot input: a 262144-body snapshot in the
               reference's own output format read by the GPU reader
               (include/g6b200_story.h), text resident on the device and from
               host bytes; the reference's get_dyn on the same text as the
               CPU baseline

Multi-GPU (torchrun, one rank per GPU): every rank integrates its own
independent cluster (different seed) -- weak scaling, no collective on the
data path; timing is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "interactions/s & %FP32 peak (acc+jerk, N=256K); p50/p99 force-call latency"
FLOPS_PER_INTERACTION = 60
N_DEFAULT = 262144
EPS2 = 1e-8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--latency-calls", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--ensemble-clusters", type=int, default=256)
    ap.add_argument("--ensemble-t", type=float, default=1.0)
    ap.add_argument("--no-grape4", action="store_true")
    ap.add_argument("--no-story", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------- plumbing
from starlab_b200.dist import Dist, cluster_seed, weak_scaling_value  # noqa: E402


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=10)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["smax"] for r in rows),
                "power_w_max": max(r["power"] for r in rows), "samples": len(rows), "reasons": sorted(reasons)}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except ValueError:
            return {}
    return {}


def traffic_from_profile():
    """DRAM bytes of one full-sweep force launch (the launch `value` times),
    from one ncu capture kept in profiles/force_sweep_traffic_n262144.json;
    None when not captured."""
    p = os.path.join(REPO, "profiles", "force_sweep_traffic_n262144.json")
    try:
        return float(json.load(open(p))["traffic_bytes_full_sweep_launch"])
    except (OSError, ValueError, KeyError):
        return None


# ---------------------------------------------------------------- workload
def make_cluster(n, seed):
    from starlab_b200 import ics
    masses = ics.salpeter_masses(n, seed + 1)
    return ics.plummer(n, seed, masses=masses)


def ensemble_section(nc, t_full, seed):
    """256 independent Plummer clusters, N log-uniform in [256, 16384],
    eps2 = (4/N)^2, eta = 0.02, mixed precision: the batched engine over one
    N-body time unit, and batched vs the plain one-call-per-cluster engine on
    the same slice [0, 1/64]."""
    from starlab_b200 import ics
    from starlab_b200.ensemble import Ensemble
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(256), np.log(16384), nc)).astype(int)
    cl = [ics.plummer(int(n), seed * 1000 + k) for k, n in enumerate(ns)]
    eps2 = (4.0 / ns) ** 2

    def make():
        return Ensemble([c[0] for c in cl], [c[1] for c in cl], [c[2] for c in cl], eps2, eta=0.02,
                        precision="mixed")

    out = {"clusters": nc, "n_total": int(ns.sum()), "n_range": [256, 16384], "eta": 0.02}
    e = make()
    e.start()
    ek0, ep0 = e.energies()
    st = e.run(t_full, tune=True)
    ek, ep = e.energies()
    de = np.abs((ek + ep) - (ek0 + ep0)) / np.abs(ek0 + ep0)
    e.close()
    out["batched_full"] = {"t_end": t_full, "seconds": st["seconds"], "interactions": st["interactions"],
                           "interactions_per_s": st["interactions"] / st["seconds"],
                           "iterations": st["iterations"], "tuned_i_tile": 256 // st["tuned_h"],
                           "tuned_tasks_per_cluster": st["tuned_tasks"],
                           "lane_efficiency": st["interactions"] / max(1, st["lane_interactions"]),
                           "dE_over_E_median": float(np.median(de)), "dE_over_E_max": float(de.max())}
    slice_t = 1.0 / 64
    for key, per in (("batched_slice", False), ("per_cluster_slice", True)):
        e = make()
        e.start()
        st = e.run(slice_t, per_cluster=per, tune=not per)
        e.close()
        out[key] = {"t_end": slice_t, "seconds": st["seconds"], "interactions": st["interactions"],
                    "interactions_per_s": st["interactions"] / st["seconds"], "iterations": st["iterations"]}
    out["speedup_vs_per_cluster"] = (out["batched_slice"]["interactions_per_s"]
                                     / out["per_cluster_slice"]["interactions_per_s"])
    return out


def served_section(seed, rates=(2000.0, 20000.0), n_calls=3000):
    """Force calls from 48 clusters (N log-uniform in [512, 65536]) arriving
    as a Poisson process, ni ~ 1/ni on [1, N]: the batching server vs the
    plain engine serving the same stream one call at a time, at the
    configured 2000 calls/s and at a rate well above what one call at a time
    can serve (the queue then builds and batches fill)."""
    from starlab_b200 import G6Engine
    from starlab_b200.server import ResidentServer, Server
    from starlab_b200.stream import make_clusters, make_stream, run_served, run_sequential
    clusters = make_clusters(48, seed)
    out = {"clusters": len(clusters), "calls": n_calls,
           "servers": {"served": "g6b200_srv_*: host dispatch lanes, one batched launch per batch",
                       "resident": "g6b200_res_*: one persistent kernel polling a request ring, no launches"}}

    def summary(lat, wall, inter, st=None):
        d = {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
             "interactions_per_s": inter / wall, "wall_s": wall}
        if st is not None:
            d.update(batches=st["batches"], mean_batch=st["requests"] / max(1, st["batches"]),
                     max_batch=st["max_batch"])
        return d

    for rate in rates:
        calls = make_stream(clusters, rate, n_calls, seed)
        row = {"rate_per_s": rate}
        for key, make in (("served", lambda: Server(precision="mixed")),
                          ("resident", lambda: ResidentServer(precision="mixed"))):
            srv = make()
            lat, wall, inter = run_served(srv, clusters, calls)
            row[key] = summary(lat, wall, inter, srv.stats())
            srv.close()
        lat2, wall2, inter2 = run_sequential(
            lambda k, n: G6Engine(cluster_id=3000 + k, precision="mixed", npipes=n), clusters, calls)
        row["one_call_at_a_time"] = summary(lat2, wall2, inter2)
        for key in ("served", "resident"):
            row[key + "_over_plain"] = row[key]["interactions_per_s"] / row["one_call_at_a_time"]["interactions_per_s"]
        out["rate_%d" % int(rate)] = row
    return out


def grape4_section(seed, n=65536, sweeps=3):
    from starlab_b200 import ics
    from starlab_b200.grape4 import H3Engine
    m, x, v = ics.plummer(n, seed)
    z = np.zeros((n, 3))
    h3 = H3Engine()
    npipe = h3.npipe()
    h3.set_j_particles(x, v, z, z, m, 0.0)
    h3.setti(0.0)

    def sweep():
        for i0 in range(0, n, npipe):
            h3.calc(n, x[i0:i0 + npipe], v[i0:i0 + npipe], 0.0, 0.0)

    sweep()
    s0 = h3.stats()
    t0 = time.perf_counter()
    for _ in range(sweeps):
        sweep()
    sec = (time.perf_counter() - t0) / sweeps
    s1 = h3.stats()
    h3.close()
    inter = n * (n - 1)
    return {"n": n, "npipe": npipe, "precision": "fp64", "ms_per_sweep": sec * 1e3,
            "interactions_per_s": inter / sec, "calls_per_sweep": (s1["calls"] - s0["calls"]) // sweeps,
            "launches_per_sweep": (s1["launches"] - s0["launches"]) // sweeps,
            "path": "h3mjpdma_indirect_/h3calc_ (host buffers, wall clock)"}


def story_section(seed, n=262144, reps=10, cpu=True):
    """Story-format snapshot input: a flat n-body snapshot (root + n leaves,
    "%.18g" numbers as the reference's put_node writes them) read through the
    reader's C ABI; the reference's own get_dyn on the same text as the CPU
    baseline (oracle/_ref/story_ref, one core)."""
    import torch
    from starlab_b200 import ics
    from starlab_b200.story import StoryReader, format_story
    m = ics.salpeter_masses(n, seed)
    _, x, v = ics.plummer(n, seed + 1, masses=m)
    text = format_story(m, x + 1e-3, v - 5e-4, log_lines=[" ===>  bench snapshot"])
    rd = StoryReader()
    d = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    out = {"n": n, "bytes": len(text), "workload": "flat snapshot, root + %d leaves, Plummer/Salpeter" % n}
    for raw in (False, True):
        for _ in range(3):
            rd.parse_device(d.data_ptr(), d.numel(), raw=raw)
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            info = rd.parse_device(d.data_ptr(), d.numel(), raw=raw)
            ts.append(time.perf_counter() - t0)
        sec = statistics.median(ts)
        out["device_raw" if raw else "device"] = {"ms": sec * 1e3, "particles_per_s": n / sec,
                                                 "text_gbs": len(text) / sec / 1e9}
    hbm = float(measured_peaks().get("hbm_gbs", 6650.0))
    out["roofline"] = {"bound": "per-line serial parsing (not HBM)", "achieved_text_gbs": out["device_raw"]["text_gbs"],
                       "peak_hbm_gbs": hbm, "frac": out["device_raw"]["text_gbs"] / hbm,
                       "peak_source": "MEASURED_PEAKS.json" if measured_peaks() else "fallback"}
    rd.leaves(rd.parse_info(text))  # warm-up: the first host-text parse allocates the pinned staging slots
    ts = []
    for _ in range(max(3, reps // 2)):
        t0 = time.perf_counter()
        info = rd.parse_info(text)
        lm, lx, lv = rd.leaves(info)
        ts.append(time.perf_counter() - t0)
    sec = statistics.median(ts)
    out["e2e"] = {"ms": sec * 1e3, "particles_per_s": n / sec, "h2d_bytes": len(text), "d2h_bytes": 56 * n,
                  "path": "g6b200_story_parse (host bytes) + g6b200_story_leaves"}
    if cpu:
        from oracle.oracle import STORY_REF, StoryOracle, ref_story_seconds
        o = StoryOracle().parse(text)
        out["matches_oracle"] = bool(np.array_equal(o.leaves_pos.view(np.uint64), lx.view(np.uint64)) and
                                     np.array_equal(o.leaves_vel.view(np.uint64), lv.view(np.uint64)) and
                                     np.array_equal(o.leaves_mass.view(np.uint64), lm.view(np.uint64)))
        if os.path.exists(STORY_REF):
            with tempfile.NamedTemporaryFile(suffix=".snap") as f:
                f.write(text)
                f.flush()
                secs = ref_story_seconds(f.name)
            out["cpu_baseline"] = {"value": n / secs, "unit": "particles/s", "cores": 1, "kind": "reference",
                                   "seconds": secs, "sample": "the same snapshot read by get_dyn"}
    rd.close()
    return out


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1) if a.ndim == 2 else np.abs(a - b) / np.abs(b)


def cpu_baseline(n, seed, cores, per_core=640, gpu=None, state=None):
    """Starlab's FP64 force loop on a bounded sample of i (rank 0, N=1):
    per_core i-particles per host thread against all N j, every particle
    first predicted to the block time by the reference's predict_loworder.
    `state` = (acc, jerk, ti): the j-state's acc and jerk (tj = 0) and the
    block time of a timed step (default: zero acc and jerk, ti = 0).  When
    `gpu` holds the engine's (acc, jerk, pot, nn) for every particle at that
    step, the reference's results for the sample also score them:
    per-particle relative error of acc, jerk and pot, nn mismatches."""
    m, x, v = make_cluster(n, seed)
    z = np.zeros((n, 3))
    a0, j0, ti = state if state is not None else (z, z, 0.0)
    try:
        from oracle.oracle import RefForce
        ref = RefForce()
        ni = int(min(n, per_core * cores))
        ilist = np.linspace(0, n - 1, ni).astype(np.int32)
        out = ref.force(m, x, v, a0, j0, 0.0, ti, float(np.sqrt(EPS2)), ilist=ilist, nthreads=cores)
        secs = out["seconds"]
        res = {"value": ni * (n - 1) / secs, "unit": "interactions/s", "cores": cores, "kind": "reference",
               "sample": "%d i (evenly spaced) x %d j, hdyn::flat_calculate_acc_and_jerk on %d threads; "
                         "force loop %.2f s" % (ni, n, cores, secs),
               "sample_i": int(ni), "sample_seconds": secs}
        if gpu is not None:
            acc, jerk, pot, nn = (g[ilist] for g in gpu)
            acc_err, jerk_err, pot_err = _rel(acc, out["acc"]), _rel(jerk, out["jerk"]), _rel(pot, out["pot"])
            res["accuracy_vs_reference"] = {
                "sample_i": int(ni), "precision": "mixed", "ti": ti,
                "step": "the last timed step: j predicted from tj = 0 to ti with the step's acc/2 and jerk/6",
                "acc": {"median": float(np.median(acc_err)), "max": float(acc_err.max())},
                "jerk": {"median": float(np.median(jerk_err)), "max": float(jerk_err.max())},
                "pot": {"median": float(np.median(pot_err)), "max": float(pot_err.max())},
                "nn_mismatch": int(np.sum(nn != out["nn"]))}
        return res
    except ImportError:
        from oracle.oracle import G6Oracle
        o = G6Oracle()
        ni = 256
        idx = np.arange(ni, dtype=np.int32)
        t0 = time.perf_counter()
        o.force(x, v, m, idx, x[:ni], v[:ni], EPS2)
        secs = time.perf_counter() - t0
        return {"value": ni * (n - 1) / secs, "unit": "interactions/s", "cores": 1, "kind": "port",
                "sample": "%d i x %d j, oracle C restatement, 1 thread" % (ni, n),
                "sample_i": ni, "sample_seconds": secs}


def accuracy_vs_fp64(m, x, v, acc, jerk, ti, got):
    """Every particle of the timed step (mixed) against the engine's FP64
    mode on the same state (FP64 prediction, pair sums and accumulation;
    pinned to <= 1e-12 of the FP64 oracle by the parity tests): per-quantity
    median / 99.9th percentile / max relative error over all i."""
    from starlab_b200 import G6Engine
    n = len(m)
    e64 = G6Engine(cluster_id=7, precision="fp64", npipes=n)
    e64.set_j_particles(0.0, m, jerk / 6.0, 0.5 * acc, v, x)
    e64.set_ti(ti)
    ref = e64.sweep(n, eps2=EPS2)
    e64.close()
    out = {"all_i": int(n), "ti": ti, "precision": "mixed vs fp64 engine"}
    for k, g, r, tol in (("acc", got[0], ref[0], 1e-6), ("jerk", got[1], ref[1], 1e-5), ("pot", got[2], ref[2], 1e-6)):
        e = _rel(g, r)
        out[k] = {"median": float(np.median(e)), "p999": float(np.quantile(e, 0.999)), "max": float(e.max()),
                  "over_tolerance": int((e > tol).sum()), "tolerance": tol}
    out["nn_mismatch"] = int(np.sum(got[3] != ref[3]))
    return out


def run_reference(args, dist):
    """--impl reference: the reference's own CPU force path, same metric."""
    if dist.rank != 0:
        return
    cores = os.cpu_count() or 1
    n = args.n
    vals, secs = [], []
    last = None
    for k in range(args.warmup + args.steps):
        r = cpu_baseline(n, 11, cores, per_core=96)
        if k >= args.warmup:
            vals.append(r["value"])
            secs.append(r.get("sample_seconds", 0.0))
        last = r
    value = statistics.median(vals)
    # A step is one bounded sample (sample_i i against all N j): ms_per_step
    # is its measured time; the full sweep's time is extrapolated from the
    # rate and labelled as such.
    per_step_ms = statistics.median(secs) * 1e3
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "interactions/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step_ms,
            "step": "sample of %d i x %d j (of the %d-i sweep)" % (last["sample_i"], n, n),
            "extrapolated": {"full_sweep_ms": n * (n - 1) / value * 1e3, "from_sample_i": last["sample_i"],
                             "note": "the full 262144 x 262143 sweep on the CPU is extrapolated linearly "
                                     "from the sample rate, not run"},
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_of(args, n),
            "cpu_baseline": {"value": value, "unit": "interactions/s", "cores": last["cores"], "kind": last["kind"],
                             "sample": last["sample"]},
            "e2e": {"value": value, "unit": "interactions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_of(args, n):
    return {"workload": "full force sweep (predict + acc/jerk/pot/nn on all i from all j), "
                        "N=%d Plummer + Salpeter masses (slope -2.35, 0.1-100), eps2=1e-8, mixed precision" % n,
            "n": n, "eps2": EPS2, "precision": "mixed (fixed-point positions, FP32 pairs, FP64 sums)",
            "interactions_per_step": n * (n - 1), "parallelism": "independent cluster per GPU",
            "l2": "256 MiB buffer written before every timed step (value); e2e re-uploads j and i from host "
                  "memory every step"}


# ---------------------------------------------------------------- sub-modes
# Bounded workloads to run under a profiler (ncu) with one command line, and
# the energy-drift measurement:
#   python bench.py profile-case --n 262144 --ni 16384 --mode mixed --calls 3
#   python bench.py profile-ensemble --t 0.015625
#   python bench.py profile-story --n 262144 --reps 3
#   python bench.py energy-drift --n 262144 --t 1
def profile_case(argv):
    """A few force calls of one shape through the C ABI: an N-particle
    Plummer/Salpeter cluster in j-memory, then `calls` firsthalf/lasthalf2
    pairs of ni i-particles at new block times (every call runs the predictor
    and the force kernel); prints the engine's device times per call."""
    ap = argparse.ArgumentParser(prog="bench.py profile-case")
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--ni", type=int, default=16384)
    ap.add_argument("--mode", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--eps2", type=float, default=1e-8)
    ap.add_argument("--h2", type=float, default=0.0)
    ap.add_argument("--config", default="", help="il,r,warps,h,nsplit")
    a = ap.parse_args(argv)
    os.environ.setdefault("G6B200_EVENT_TIMING", "1")  # per-call device times in the stats
    from starlab_b200 import G6Engine, ics
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
    return 0


def profile_ensemble(argv):
    """One slice of the bench's ensemble workload (256 Plummer clusters, N
    log-uniform in [256, 16384], seed 2024, eps^2 = (4/N)^2, eta = 0.02,
    mixed), from t = 0 to --t; prints the run's statistics."""
    ap = argparse.ArgumentParser(prog="bench.py profile-ensemble")
    ap.add_argument("--clusters", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--t", type=float, default=1.0 / 64)
    ap.add_argument("--tune", action="store_true")
    a = ap.parse_args(argv)
    from starlab_b200 import ics
    from starlab_b200.ensemble import Ensemble
    rng = np.random.default_rng(a.seed)
    ns = np.exp(rng.uniform(np.log(256), np.log(16384), a.clusters)).astype(int)
    cl = [ics.plummer(int(n), a.seed * 1000 + k) for k, n in enumerate(ns)]
    e = Ensemble([c[0] for c in cl], [c[1] for c in cl], [c[2] for c in cl], (4.0 / ns) ** 2, eta=0.02,
                 precision="mixed")
    e.start()
    st = e.run(a.t, tune=a.tune)
    e.close()
    st["interactions_per_s"] = st["interactions"] / st["seconds"]
    st["us_per_iteration"] = st["seconds"] / st["iterations"] * 1e6
    st["lane_efficiency"] = st["interactions"] / max(1, st["lane_interactions"])
    print(json.dumps(st))
    return 0


def profile_story(argv):
    """A flat N-body snapshot in the reference's output format, resident in
    device memory, parsed --reps times corrected and --reps times raw;
    prints the median wall time of each."""
    ap = argparse.ArgumentParser(prog="bench.py profile-story")
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=11)
    a = ap.parse_args(argv)
    import torch
    from starlab_b200 import ics
    from starlab_b200.story import StoryReader, format_story
    m = ics.salpeter_masses(a.n, a.seed)
    _, x, v = ics.plummer(a.n, a.seed + 1, masses=m)
    text = format_story(m, x + 1e-3, v - 5e-4)
    d = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    rd = StoryReader()
    for raw in (False, True):
        ts = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            info = rd.parse_device(d.data_ptr(), d.numel(), raw=raw)
            ts.append(time.perf_counter() - t0)
        print("raw=%d n=%d bytes=%d nodes=%d median %.3f ms" % (raw, a.n, len(text), info.n_nodes,
                                                                 1e3 * statistics.median(ts)))
    rd.close()
    return 0


def energy_drift(argv):
    """Energy conservation at scale: one N = 262144 Plummer sphere with
    Salpeter masses (the bench's cluster), eps^2 = 1e-8, integrated from
    t = 0 to --t with the device Hermite block-step integrator (eta = 0.02)
    in the mixed and in the FP64 mode.  Energies of the initial and final
    states from the engine's FP64 potential-only sweep (g6b200_energies),
    the stand-in for the reference's hsys_stats -0 at a size where a CPU
    run is out of reach.  Prints one JSON line."""
    ap = argparse.ArgumentParser(prog="bench.py energy-drift")
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--t", type=float, default=1.0)
    ap.add_argument("--eta", type=float, default=0.02)
    ap.add_argument("--modes", default="mixed,fp64")
    a = ap.parse_args(argv)
    from starlab_b200 import G6Engine
    from starlab_b200.ensemble import Ensemble
    n = a.n
    m, x, v = make_cluster(n, 11)

    def energy(mm, xx, vv):
        e = G6Engine(cluster_id=9, precision="fp64", npipes=n)
        z = np.zeros((n, 3))
        e.set_j_particles(0.0, mm, z, z, vv, xx)
        e.set_ti(0.0)
        ep, ek = e.energies(n, EPS2)
        e.close()
        return ep + ek

    e0 = energy(m, x, v)
    out = {"n": n, "eps2": EPS2, "eta": a.eta, "t_end": a.t, "E0": e0,
           "energy_tool": "g6b200_energies, FP64 mode (potential-only sweep + device sums)"}
    for mode in a.modes.split(","):
        ens = Ensemble([m], [x], [v], EPS2, eta=a.eta, precision=mode)
        ens.start()
        st = ens.run(a.t)
        f = ens.get(0)
        ens.close()
        e1 = energy(f["m"], f["x"], f["v"])
        out[mode] = {"seconds": st["seconds"], "iterations": st["iterations"], "interactions": st["interactions"],
                     "interactions_per_s": st["interactions"] / max(st["seconds"], 1e-9),
                     "t_min": float(f["t"].min()), "t_max": float(f["t"].max()),
                     "E1": e1, "dE_over_E": abs(e1 - e0) / abs(e0)}
    if "mixed" in out and "fp64" in out:
        out["mixed_over_fp64"] = out["mixed"]["dE_over_E"] / max(out["fp64"]["dE_over_E"], 1e-300)
    print(json.dumps(out), flush=True)
    return 0


def serve(argv):
    """The served-stream section alone (48 clusters, Poisson arrivals) at
    the given rates; prints one JSON line."""
    ap = argparse.ArgumentParser(prog="bench.py serve")
    ap.add_argument("--rates", default="2000,20000")
    ap.add_argument("--calls", type=int, default=3000)
    ap.add_argument("--seed", type=int, default=5)
    a = ap.parse_args(argv)
    rates = tuple(float(r) for r in a.rates.split(","))
    print(json.dumps(served_section(a.seed, rates=rates, n_calls=a.calls)), flush=True)
    return 0


SUB_MODES = {"profile-case": profile_case, "profile-ensemble": profile_ensemble, "profile-story": profile_story,
             "energy-drift": energy_drift, "serve": serve}


def main():
    if len(sys.argv) > 1 and sys.argv[1] in SUB_MODES:
        return SUB_MODES[sys.argv[1]](sys.argv[2:])
    args = parse()
    if args.impl == "reference":
        dist = Dist(use_cuda=False)
        run_reference(args, dist)
        dist.close()
        return 0
    import torch
    dist = Dist(use_cuda=True)
    dev = dist.local
    torch.cuda.set_device(dev)
    os.environ["G6B200_DEVICE"] = str(dev)
    from starlab_b200 import G6Engine

    n = args.n
    seed = cluster_seed(11, dist.rank)
    m, x, v = make_cluster(n, seed)
    z = np.zeros((n, 3))
    eng = G6Engine(cluster_id=0, precision="mixed", npipes=n)
    # acc/jerk for the predictor from one sweep at t = 0
    eng.set_j_particles(0.0, m, z, z, v, x)
    eng.set_ti(0.0)
    acc, jerk, pot, nn = eng.sweep(n, eps2=EPS2)
    eng.set_j_particles(0.0, m, jerk / 6.0, 0.5 * acc, v, x)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    dt = 1.0 / 1024

    def device_step(k):
        flush.zero_()
        torch.cuda.synchronize()
        eng.set_ti(dt * (k + 1))
        eng.sweep(n, eps2=EPS2, copy_out=False)
        return eng.stats()

    for k in range(args.warmup):
        device_step(k)
    sampler = ClockSampler(dev)
    dist.barrier()
    torch.cuda.synchronize()
    l0 = eng.stats()["launches"]
    step_ms, force_ms, pred_ms = [], [], []
    for k in range(args.steps):
        st = device_step(args.warmup + k)
        step_ms.append(st["last_call_ms"])
        force_ms.append(st["last_force_ms"])
        pred_ms.append(st["last_predict_ms"])
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    launches = eng.stats()["launches"] - l0
    # the last timed step's results, for the accuracy checks: the same sweep
    # at the same block time, copied out
    ti_last = dt * (args.warmup + args.steps)
    eng.set_ti(ti_last)
    gpu_last = eng.sweep(n, eps2=EPS2)
    total_ms = dist.max(sum(step_ms))
    interactions = n * (n - 1)
    value = weak_scaling_value(dist.world, interactions, args.steps, total_ms)

    # ---- e2e through the C ABI with host buffers
    e2e_steps = args.e2e_steps or max(3, args.steps // 2)
    npipes = 16384
    eng2 = G6Engine(cluster_id=1, precision="mixed", npipes=npipes)
    idx = np.arange(n, dtype=np.int32)
    a2, j6 = 0.5 * acc, jerk / 6.0

    def e2e_step(k):
        ti = dt * (k + 1)
        eng2.set_j_particles(0.0, m, j6, a2, v, x)
        eng2.set_ti(ti)
        # host-side i prediction (the caller's job in kira) is outside the
        # engine; the i arrays are those of the step's block time
        res = eng2.force(n, idx, xp_h, vp_h, EPS2)
        return res

    xp_h = x + dt * (v + dt * (a2 + dt * j6))
    vp_h = v + dt * (2 * a2 + dt * 3 * j6)
    for k in range(2):
        e2e_step(k)
    s0 = eng2.stats()
    dist.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        e2e_step(k)
    t1 = time.perf_counter()
    dist.barrier()
    s1 = eng2.stats()
    e2e_s = dist.max(t1 - t0)
    e2e_value = dist.world * interactions * e2e_steps / e2e_s
    h2d = (s1["h2d_bytes"] - s0["h2d_bytes"]) / e2e_steps
    d2h = (s1["d2h_bytes"] - s0["d2h_bytes"]) / e2e_steps

    # ---- force-call latency (kira-like i-blocks on the same cluster)
    rng = np.random.default_rng(5 + dist.rank)
    lat = []
    u = rng.uniform(0, 1, args.latency_calls)
    nis = np.clip(np.exp(u * np.log(n)).astype(int), 1, n)  # p(ni) ~ 1/ni on [1, N]
    eng3 = G6Engine(cluster_id=2, precision="mixed", npipes=n)
    eng3.set_j_particles(0.0, m, j6, a2, v, x)
    eng3.set_ti(dt)
    for ni in nis[:5]:
        eng3.force(n, idx[:ni], xp_h[:ni], vp_h[:ni], EPS2)
    for ni in nis:
        s = rng.integers(0, n - ni + 1)
        t0 = time.perf_counter()
        eng3.calc_firsthalf(n, idx[s:s + ni], xp_h[s:s + ni], vp_h[s:s + ni], EPS2)
        eng3.calc_lasthalf2()
        lat.append((time.perf_counter() - t0) * 1e3)
    lat = np.array(lat)

    if dist.rank == 0:
        props = torch.cuda.get_device_properties(dev)
        peaks = measured_peaks()
        sm_max = float(peaks.get("sm_max_mhz", 1965.0))
        sms = props.multi_processor_count
        nominal_tflops = sms * 128 * 2 * sm_max * 1e6 / 1e12
        # the FP32 FMA rate measured on this GPU, after the timed region
        import ctypes
        from starlab_b200 import load_library
        lib = load_library()
        lib.g6b200_measure_fp32_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        measured = ctypes.c_double(0)
        peak_ok = lib.g6b200_measure_fp32_peak(dev, ctypes.byref(measured)) == 0 and measured.value > 0
        peak_tflops = measured.value if peak_ok else nominal_tflops
        mean_force = statistics.mean(force_ms)
        achieved = FLOPS_PER_INTERACTION * interactions / (mean_force * 1e-3) / 1e12
        traffic = traffic_from_profile()
        line = {
            "metric": METRIC, "value": value, "unit": "interactions/s", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config_of(args, n),
            "gflops": value * FLOPS_PER_INTERACTION / 1e9,
            "fp32_peak_frac": achieved / peak_tflops,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
                         "frac": achieved / peak_tflops, "traffic": traffic,
                         "kernel": "force_kernel (mixed, + split reduction)",
                         "force_ms_mean": mean_force, "predict_ms_mean": statistics.mean(pred_ms),
                         "peak_source": ("measured in this run: packed FP32x2 FMA chains on every SM "
                                         "(g6b200_measure_fp32_peak)" if peak_ok else
                                         "derived (measurement failed)"),
                         "peak_nominal": nominal_tflops,
                         "peak_nominal_source": "%d SMs x 128 FP32 lanes x 2 flops x %.0f MHz (max SM clock%s)"
                                                % (sms, sm_max, ", MEASURED_PEAKS.json" if peaks else ", fallback")},
            "e2e": {"value": e2e_value, "unit": "interactions/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps, "npipes": npipes,
                    "ms_per_step": e2e_s / e2e_steps * 1e3},
            "latency": {"unit": "ms", "calls": int(len(lat)), "p50": float(np.percentile(lat, 50)),
                        "p99": float(np.percentile(lat, 99)),
                        "ni_distribution": "power law slope -1 on [1, N]", "path": "g6calc_firsthalf_/lasthalf2_"},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if dist.world == 1 and not args.no_ensemble:
            line["ensemble"] = ensemble_section(args.ensemble_clusters, args.ensemble_t, 2024)
        if dist.world == 1 and not args.no_served:
            line["served_stream"] = served_section(5)
        if dist.world == 1 and not args.no_grape4:
            line["grape4"] = grape4_section(7)
        if dist.world == 1 and not args.no_story:
            line["story"] = story_section(11, cpu=not args.no_cpu_baseline)
        if dist.world == 1:
            line["accuracy_vs_fp64_engine"] = accuracy_vs_fp64(m, x, v, acc, jerk, ti_last, gpu_last)
        if dist.world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(n, seed, os.cpu_count() or 1, gpu=gpu_last,
                                                state=(acc, jerk, ti_last))
        print(json.dumps(line), flush=True)
    for e in (eng, eng2, eng3):
        e.close()
    dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
