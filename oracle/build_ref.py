#!/usr/bin/env python3
"""Build recipe for the reference oracle (test infrastructure, not product).

Compiles Starlab's own FP64 CPU force path from the read-only reference tree
with g++ directly (no autotools: they are absent here), into ``oracle/_ref/``:

* ``libstarlab.a``    every ``lib*_la_SOURCES`` file of the directories kira
                       links (``src/std``, ``src/node/...``, ``src/star/...``),
                       minus the GRAPE stubs, the bison/flex reader and the
                       Fortran ``nstab.f`` (no gfortran; replaced by
                       ``oracle/nstab_stub.c``);
* ``libstubs.a``       the reference's GRAPE-4/GRAPE-6 null stubs
                       (``src/node/dyn/hdyn/stubs/grape6_stubs.c``), linked
                       last exactly as ``evolve/Makefile.am:36-48`` does;
* tools               ``kira``, ``makeplummer``, ``makemass``, ``scale``,
                       ``makesecondary``, ``makebinary`` (primordial binaries),
                       ``hsys_stats``, ``hscale`` (TOOLBOX mains, CPU engine);
* ``kira_g6``/``hsys_stats_g6``  the same mains linked against
                       ``libg6b200.so`` before the stubs, i.e. the unchanged
                       caller driving the GPU engine through the g6 ABI
                       (built only when the engine library exists);
* ``story_ref``         ``oracle/story_ref.C``: the reference's snapshot
                       reader (``get_dyn``) run on a story text, every node
                       printed exactly (hex floats), or ``-t``: its time;
* ``libref_force.so``  ``oracle/ref_force.C``: a C entry point over the
                       reference's ``predict_loworder`` and
                       ``hdyn::flat_calculate_acc_and_jerk``
                       (``src/node/dyn/hdyn/evolve/hdyn_ev.C:2047``);
* ``libharp3sim.so``   the reference's IEEE GRAPE-4 simulator
                       (``src/harpsims/harp3fastsim.c``), compiled as it is
                       (K&R C: ``-std=gnu89``), the executable definition of
                       the GRAPE-4 ABI;
* ``kira_g4``/``hsys_stats_g4``  the mains linked against ``libh3b200.so``,
                       with ``hdyn_grape4.C`` recompiled under
                       ``USE_HALF_CHIP`` as configure defines it when it finds
                       a GRAPE-4 library (``configure.ac:216-222``);
* ``kira_g4o``/``hsys_stats_g4o``  the same GRAPE-4 branch on the CPU, over
                       ``oracle/h3_oracle.c`` + ``oracle/g4_oracle.c`` (the
                       GRAPE-4 ABI on the oracle's pipeline restatement);
* ``kira_g6o``/``hsys_stats_g6o``/``hscale_g6o``/``get_densities_g6o``  the
                       GRAPE-6 branch on the CPU, over
                       ``oracle/g6_abi_oracle.c`` + ``oracle/g6_oracle.c``.

Nothing here is shipped; the outputs are git-ignored.  Usage:
``python oracle/build_ref.py [--jobs N] [--ref PATH]``.
"""
import argparse
import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")

# Directories whose libtool convenience libraries kira links (the set its Makefile.am files name).
LIB_DIRS = [
    "std", "node/util", "node/dyn/util", "node/dyn/kepler", "node/dyn/init",
    "node/dyn/evolve", "node/dyn/_dyn_", "node/dyn/hdyn/util",
    "node/dyn/hdyn/evolve", "node/dyn/hdyn/xutil",
    "star/dstar/init", "star/dstar/io", "star/dstar/starclass",
    "star/dstar/stardyn", "star/dstar/util",
    "star/sstar/init", "star/sstar/io", "star/sstar/starclass",
    "star/sstar/stardyn", "star/util",
]
# Sources dropped from the library: generated reader (unused by kira; the
# lexer needs an undefined symbol) and Fortran (no compiler in the image).
DROP = {"dyn_parser.yy", "dyn_lexer.ll", "nstab.f", "pp3_widget.C",
        "moc_pp3_widget.C"}
STUB_FILES = ["node/dyn/hdyn/stubs/grape4_stubs.c",
              "node/dyn/hdyn/stubs/grape6_stubs.c",
              "node/dyn/hdyn/stubs/sapporo_stubs.c"]
TOOLS = {
    "kira": "node/dyn/hdyn/evolve/kira.C",
    "makeplummer": "node/dyn/init/makeplummer.C",
    "makemass": "node/util/makemass.C",
    "scale": "node/dyn/util/scale.C",
    "hsys_stats": "node/dyn/hdyn/util/hsys_stats.C",
    "hscale": "node/dyn/hdyn/util/hscale.C",
    "get_densities": "node/dyn/hdyn/util/get_densities.C",
    "compute_density": "node/dyn/util/compute_density.C",
    "makesecondary": "node/dyn/util/makesecondary.C",
    "makebinary": "node/dyn/init/makebinary.C",
}
CONFIG_H = """/* hand-written stand-in for the autoconf config.h of Starlab 4.4.4 */
#define HAVE_LIBPTHREAD 1
#define HAVE_STDBOOL_H 1
#define HAVE_STPCPY 1
#define F77_FUNC(name,NAME) name ## _
#define STARLAB_VERSION "4.4.4"
#define VERSION "4.4.4"
#define PACKAGE "starlab"
"""


def parse_la_sources(makefile_am):
    """Return the file names listed in every ``lib*_la_SOURCES`` of a Makefile.am."""
    text = open(makefile_am).read().replace("\\\n", " ")
    files = []
    for m in re.finditer(r"^\s*lib\S*_la_SOURCES\s*\+?=(.*)$", text, re.M):
        files += m.group(1).split()
    return files


def run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout[-4000:]))
    return r.stdout


def up_to_date(out, srcs):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in srcs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("STARLAB_REFERENCE"),
                    help="root of the reference source tree (or STARLAB_REFERENCE); required")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--quiet", action="store_true")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or STARLAB_REFERENCE) must name the reference source tree")
    src = os.path.join(args.ref, "src")
    if not os.path.isdir(src):
        print("reference tree not found at %s; skipping oracle/_ref build" % args.ref)
        return 0
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    os.makedirs(os.path.join(OUT, "include"), exist_ok=True)
    cfg = os.path.join(OUT, "include", "config.h")
    if not os.path.exists(cfg) or open(cfg).read() != CONFIG_H:
        open(cfg, "w").write(CONFIG_H)

    inc = ["-I" + os.path.join(OUT, "include"), "-I" + os.path.join(args.ref, "include"),
           "-I" + os.path.join(args.ref, "include", "star")]
    cxx = ["g++", "-std=gnu++98", "-fpermissive", "-O2", "-fPIC", "-w",
           "-DHAVE_CONFIG_H", "-D_SRC_=\"starlab\""] + inc
    cc = ["gcc", "-O2", "-fPIC", "-w", "-DHAVE_CONFIG_H"] + inc

    jobs = []   # (obj, cmd, deps)

    def add(srcfile, obj, extra=(), c=False):
        base = cc if c else cxx
        jobs.append((obj, base + list(extra) + ["-c", srcfile, "-o", obj], [srcfile, cfg]))

    lib_objs = []
    for d in LIB_DIRS:
        mk = os.path.join(src, d, "Makefile.am")
        for f in parse_la_sources(mk):
            if f in DROP or not (f.endswith(".C") or f.endswith(".c")):
                continue
            if d == "node/dyn/hdyn/xutil" and f != "Qt_pp3.C":
                continue
            obj = os.path.join(OUT, "obj", d.replace("/", "_") + "__" + f + ".o")
            add(os.path.join(src, d, f), obj, c=f.endswith(".c"))
            lib_objs.append(obj)
    nstab_obj = os.path.join(OUT, "obj", "nstab_stub.o")
    add(os.path.join(HERE, "nstab_stub.c"), nstab_obj, c=True)
    lib_objs.append(nstab_obj)
    stub_objs = []
    for f in STUB_FILES:
        obj = os.path.join(OUT, "obj", "stubs__" + os.path.basename(f) + ".o")
        add(os.path.join(src, f), obj, c=True)
        stub_objs.append(obj)
    tool_objs = {}
    for name, f in TOOLS.items():
        obj = os.path.join(OUT, "obj", "tool__" + name + ".o")
        add(os.path.join(src, f), obj, extra=["-DTOOLBOX"])
        tool_objs[name] = obj
    harness_obj = os.path.join(OUT, "obj", "ref_force.o")
    add(os.path.join(HERE, "ref_force.C"), harness_obj)
    story_obj = os.path.join(OUT, "obj", "story_ref.o")
    add(os.path.join(HERE, "story_ref.C"), story_obj)
    g4_obj = os.path.join(OUT, "obj", "hdyn_grape4_half_chip.o")
    add(os.path.join(src, "node/dyn/hdyn/evolve/hdyn_grape4.C"), g4_obj, extra=["-DUSE_HALF_CHIP=1"])
    oobj = {}
    for f in ("h3_oracle.c", "g4_oracle.c", "g6_abi_oracle.c", "g6_oracle.c"):
        oobj[f] = os.path.join(OUT, "obj", "oracle__" + f + ".o")
        add(os.path.join(HERE, f), oobj[f], extra=["-ffp-contract=off"], c=True)
    h3o_objs = [oobj["h3_oracle.c"], oobj["g4_oracle.c"]]
    g6o_objs = [oobj["g6_abi_oracle.c"], oobj["g6_oracle.c"]]
    sim_src = os.path.join(src, "harpsims", "harp3fastsim.c")
    sim_obj = os.path.join(OUT, "obj", "harp3fastsim.o")
    add(sim_src, sim_obj, extra=["-std=gnu89"], c=True)

    todo = [j for j in jobs if not up_to_date(j[0], j[2])]
    if not args.quiet:
        print("oracle/_ref: compiling %d of %d sources with %d jobs" % (len(todo), len(jobs), args.jobs))
    with cf.ThreadPoolExecutor(args.jobs) as ex:
        list(ex.map(lambda j: run(j[1]), todo))

    lib = os.path.join(OUT, "libstarlab.a")
    if not up_to_date(lib, lib_objs):
        if os.path.exists(lib):
            os.remove(lib)
        run(["ar", "rcs", lib] + lib_objs)
    stubs = os.path.join(OUT, "libstubs.a")
    if not up_to_date(stubs, stub_objs):
        if os.path.exists(stubs):
            os.remove(stubs)
        run(["ar", "rcs", stubs] + stub_objs)

    link_tail = ["-Wl,--allow-multiple-definition", "-lpthread", "-lm"]
    for name, obj in tool_objs.items():
        exe = os.path.join(OUT, name)
        if not up_to_date(exe, [obj, lib, stubs]):
            run(["g++", "-o", exe, obj, lib, stubs] + link_tail)
    exe = os.path.join(OUT, "story_ref")
    if not up_to_date(exe, [story_obj, lib, stubs]):
        run(["g++", "-o", exe, story_obj, lib, stubs] + link_tail)
    so = os.path.join(OUT, "libref_force.so")
    if not up_to_date(so, [harness_obj, lib, stubs]):
        run(["g++", "-shared", "-o", so, harness_obj, "-Wl,--whole-archive", lib,
             "-Wl,--no-whole-archive", stubs] + link_tail)

    sim_so = os.path.join(OUT, "libharp3sim.so")
    if not up_to_date(sim_so, [sim_obj]):
        run(["gcc", "-shared", "-o", sim_so, sim_obj, "-lm"])

    # kira and hsys_stats, GRAPE-4 branch, over the CPU oracle pipeline.
    for name in ("kira", "hsys_stats", "get_densities"):
        exe = os.path.join(OUT, name + "_g4o")
        if not up_to_date(exe, [tool_objs[name], g4_obj, lib, stubs] + h3o_objs):
            run(["g++", "-o", exe, tool_objs[name], g4_obj, lib] + h3o_objs + [stubs] + link_tail)

    # ... and their GRAPE-6 branch over the CPU oracle.
    for name in ("kira", "hsys_stats", "hscale", "get_densities"):
        exe = os.path.join(OUT, name + "_g6o")
        if not up_to_date(exe, [tool_objs[name], lib, stubs] + g6o_objs):
            run(["g++", "-o", exe, tool_objs[name], lib] + g6o_objs + [stubs] + link_tail)

    # kira and hsys_stats driving the GPU engine through the unchanged g6 ABI.
    g6lib_dir = os.path.join(REPO, "starlab_b200", "lib")
    g6lib = os.path.join(g6lib_dir, "libg6b200.so")
    if os.path.exists(g6lib):
        rpath = "-Wl,-rpath,$ORIGIN/../../starlab_b200/lib"
        for name in ("kira", "hsys_stats", "hscale", "get_densities"):
            exe = os.path.join(OUT, name + "_g6")
            if not up_to_date(exe, [tool_objs[name], lib, stubs, g6lib]):
                run(["g++", "-o", exe, tool_objs[name], lib, "-L" + g6lib_dir, "-lg6b200",
                     rpath, stubs] + link_tail)
    # The same mains on the GRAPE-4 ABI (kira's config == 1 branch).
    h3lib = os.path.join(g6lib_dir, "libh3b200.so")
    if os.path.exists(h3lib):
        rpath = "-Wl,-rpath,$ORIGIN/../../starlab_b200/lib"
        for name in ("kira", "hsys_stats", "hscale", "get_densities"):
            exe = os.path.join(OUT, name + "_g4")
            if not up_to_date(exe, [tool_objs[name], g4_obj, lib, stubs, h3lib]):
                run(["g++", "-o", exe, tool_objs[name], g4_obj, lib, "-L" + g6lib_dir, "-lh3b200",
                     rpath, stubs] + link_tail)
    if not args.quiet:
        print("oracle/_ref: done")
    return 0


if __name__ == "__main__":
    sys.exit(main())
