"""Build the engine library and the oracle's C restatement in-tree.

* ``starlab_b200/lib/libg6b200.so`` -- every ``csrc/*.cu`` but ``grape4.cu``
  compiled by nvcc for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``),
  linked as one shared library exporting the C ABI of ``include/g6b200.h``.
* ``starlab_b200/lib/libh3b200.so`` -- the GRAPE-4 ABI of ``include/h3b200.h``:
  ``grape4.cu`` with the engine objects it drives (a library of its own, since
  kira takes its GRAPE-4 branch whenever ``h3npipe_()`` answers).
* ``oracle/_build/libg6oracle.so`` / ``libg4oracle.so`` / ``libstoryoracle.so``
  -- the oracle's C restatements ``oracle/g6_oracle.c``, ``oracle/g4_oracle.c``
  and ``oracle/story_oracle.c`` (test infrastructure) with gcc, FP
  contraction off.

Usage: ``python -m starlab_b200.build [--verbose] [--ptxas-v]``.
"""
import argparse
import os
import subprocess
import sys
import concurrent.futures as cf

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(PKG, "_build")
LIB = os.path.join(LIBDIR, "libg6b200.so")
LIB_H3 = os.path.join(LIBDIR, "libh3b200.so")
H3_ONLY = {"grape4.o"}
H3_OBJS = {"engine.o", "force.o", "predict.o", "nblist.o", "energy.o", "split.o", "refine.o", "grape4.o"}
ORACLE_SRC = os.path.join(REPO, "oracle", "g6_oracle.c")
ORACLE_LIB = os.path.join(REPO, "oracle", "_build", "libg6oracle.so")
ORACLE_G4_SRC = os.path.join(REPO, "oracle", "g4_oracle.c")
ORACLE_G4_LIB = os.path.join(REPO, "oracle", "_build", "libg4oracle.so")
ORACLE_STORY_SRC = os.path.join(REPO, "oracle", "story_oracle.c")
ORACLE_STORY_LIB = os.path.join(REPO, "oracle", "_build", "libstoryoracle.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include")]


def _newer(out, deps):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s" % (" ".join(cmd), r.stdout))
    if verbose and r.stdout.strip():
        print(r.stdout)
    return r.stdout


def build_engine(verbose=False, ptxas_v=False, force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(REPO, "include", "g6b200.h"))
    headers.append(os.path.join(REPO, "include", "h3b200.h"))
    headers.append(os.path.join(REPO, "include", "g6b200_story.h"))
    objs, jobs = [], []
    for f in srcs:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJDIR, f[:-3] + ".o")
        objs.append(obj)
        if force or not _newer(obj, [src] + headers):
            cmd = [NVCC] + ARCH + NVFLAGS + (["-Xptxas", "-v"] if ptxas_v else []) + ["-c", src, "-o", obj]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        outs = list(ex.map(lambda c: _run(c, verbose), jobs))
    if ptxas_v:
        for o in outs:
            print(o)
    g6_objs = [o for o in objs if os.path.basename(o) not in H3_ONLY]
    h3_objs = [o for o in objs if os.path.basename(o) in H3_OBJS]
    if force or jobs or not _newer(LIB, g6_objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + g6_objs + ["-lcudart"], verbose)
    if force or jobs or not _newer(LIB_H3, h3_objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB_H3] + h3_objs + ["-lcudart"], verbose)
    return LIB


def build_oracle(verbose=False):
    os.makedirs(os.path.dirname(ORACLE_LIB), exist_ok=True)
    for src, lib in ((ORACLE_SRC, ORACLE_LIB), (ORACLE_G4_SRC, ORACLE_G4_LIB), (ORACLE_STORY_SRC, ORACLE_STORY_LIB)):
        if not _newer(lib, [src]):
            _run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-o", lib, src, "-lm"], verbose)
    return ORACLE_LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    build_engine(a.verbose, a.ptxas_v, a.force)
    build_oracle(a.verbose)
    print("built", LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main())
