"""Story-format test texts for the snapshot reader (shared by the CPU and GPU
tests and the golden-fixture script).

* ``flat_text``         -- a root and n leaves, as put_node writes one
  (starlab_b200.story.format_story), Salpeter masses, centre of mass off the
  origin so that check_and_correct_node moves every leaf;
* ``hierarchy_text``    -- several snapshots of nested binaries and triples
  with Log stories holding chapters, Star/Hydro sections, extra Dynamics keys
  the dyn reader keeps as story text, names, repeated keys (the last wins),
  missing fields (defaults), root system times, and numbers in every form
  strtod reads (exponents, signs, integers, short and long mantissas);
* ``MALFORMED``         -- texts the reference cannot read (it exits or reads
  past its buffer) or that this reader rejects; each must give an error;
* ``VARIANTS``          -- small valid texts at the corners of the reference
  reader's rules: a Dynamics section after the children, repeated sections,
  blank lines, CRLF endings, tabs, chapters holding key lines inside a
  Dynamics section or a particle body, Particle-like chapters inside Log and
  Star, deep nesting, parents of zero or negative mass, every strtod /
  strtol form, lines cut at 254 characters, an unterminated last line;
* ``random_valid_text`` -- seeded random texts the reference reads without
  error (random trees and section orders, chapters, blank lines, CRLF).
"""
import numpy as np

from starlab_b200.ics import plummer, salpeter_masses
from starlab_b200.story import format_story


def flat_text(n, seed, shift=(1e-3, -2e-3, 5e-4)):
    m = salpeter_masses(n, seed)
    _, x, v = plummer(n, seed + 1, masses=m)
    x = x + np.asarray(shift)
    v = v - 0.5 * np.asarray(shift)
    return format_story(m, x, v, system_time=0.0,
                        log_lines=[" ===>  synthetic snapshot", "       seed = %d" % seed, "  initial_mass = 1"])


def _num(rng, x):
    r = rng.random()
    if r < 0.55:
        return "%.18g" % x
    if r < 0.7:
        return "%.17g" % x
    if r < 0.8:
        return "%.6e" % x
    if r < 0.88:
        return "%+.10g" % x
    if r < 0.94:
        return "%.25g" % x
    return "%.3f" % x


def _node(rng, out, depth, idx, names):
    out.append("(Particle")
    if rng.random() < 0.9:
        out.append("  i = %d" % idx[0])
    if rng.random() < 0.15:
        nm = "b%d_%d" % (depth, idx[0])
        names.append(nm)
        out.append("  name = %s" % nm)
    idx[0] += 1
    n_d = 0
    if depth < 4 and rng.random() < (0.6 if depth == 0 else 0.25):
        n_d = 2 if rng.random() < 0.8 else 3
    out.append("  N = %d" % max(n_d, 1))
    out.append("(Log")
    if rng.random() < 0.3:
        out += ["  note = log line", "(Chapter one", "  inner = 1", "(sub", "  deeper", ")sub", ")Chapter one"]
    out.append(")Log")
    out.append("(Dynamics")
    m = float(rng.uniform(0.1, 2.0))
    x = rng.normal(size=3) * 10.0 ** rng.integers(-6, 2)
    v = rng.normal(size=3)
    if rng.random() < 0.9:
        out.append("  m  =  " + _num(rng, m))
    if rng.random() < 0.9:
        out.append("  r  =  " + " ".join(_num(rng, c) for c in x))
    if rng.random() < 0.9:
        out.append("  v  =  " + " ".join(_num(rng, c) for c in v))
    if rng.random() < 0.3:
        out.append("  a  =  1 2 3")
        out.append("  pot  =  -0.5")
        out.append("  t  =  0.125")
    if rng.random() < 0.1:
        out.append("  m  =  " + _num(rng, m * 1.5))     # a repeated key: the last one wins
    if rng.random() < 0.05:
        out.append("  r  =  1e-3 -2E+1 +7")
    out.append(")Dynamics")
    out += ["(Hydro", ")Hydro", "(Star"]
    if depth == 0:
        out += ["  mass_scale     =  -1", "  size_scale     =  -1", "  time_scale     =  -1"]
    out.append(")Star")
    for _ in range(n_d):
        _node(rng, out, depth + 1, idx, names)
    out.append(")Particle")


def hierarchy_text(seed, roots=3, leaves_per_root=40):
    rng = np.random.default_rng(seed)
    out = []
    idx = [1]
    names = []
    for r in range(roots):
        out += ["(Particle", "  N = %d" % leaves_per_root, "(Log", " ===>  hierarchy %d" % r, ")Log", "(Dynamics"]
        if r == 1:
            out.append("  real_system_time  =  0.5")
        if r != 2:
            out.append("  system_time  =  " + _num(rng, 0.25 * (r + 1)))
        out += ["  m  =  1", "  r  =  0 0 0", "  v  =  0 0 0", ")Dynamics", "(Hydro", ")Hydro", "(Star",
                ")Star"]
        for _ in range(leaves_per_root):
            _node(rng, out, 1, idx, names)
        out.append(")Particle")
    return ("\n".join(out) + "\n").encode()


MALFORMED = {
    "unclosed particle": "(Particle\n  N = 1\n(Dynamics\n  m = 1\n)Dynamics\n",
    "top-level key line": "(Particle\n)Particle\n  m = 1\n",
    "unexpected keyword": "(Particle\n  mass = 1\n)Particle\n",
    "vector with two reals": "(Particle\n(Dynamics\n  r = 1 2\n)Dynamics\n)Particle\n",
    "log title mismatch": "(Particle\n(Log\n(abc\n)abd\n)Log\n)Particle\n",
    "empty line in a log": "(Particle\n(Log\n\n)Log\n)Particle\n",
    "long log line": "(Particle\n(Log\n  " + "x" * 300 + "\n)Log\n)Particle\n",
    "stray close at top": ")Particle\n",
    "NUL byte": "(Particle\n  i = 1\x00\n)Particle\n",
}


def _leaf(i, m, r, v, extra=()):
    return ["(Particle", "  i = %d" % i, "  N = 1", "(Log", ")Log", "(Dynamics", "  m  =  %s" % m,
            "  r  =  %s" % r, "  v  =  %s" % v] + list(extra) + [")Dynamics", "(Hydro", ")Hydro", "(Star", ")Star",
                                                                 ")Particle"]


def _root(children, head=()):
    return ["(Particle", "  N = 2", "(Log", ")Log", "(Dynamics", "  system_time  =  0.5", "  m  =  1",
            "  r  =  0 0 0", "  v  =  0 0 0", ")Dynamics"] + list(head) + children + [")Particle"]


def _j(lines, nl="\n"):
    return (nl.join(lines) + nl).encode()


# Valid texts that exercise the corners of the reference reader's rules.
VARIANTS = {
    "dynamics after children": _j(["(Particle", "  i = 10"] + _leaf(1, "0.25", "1 0 0", "0 1 0") +
                                  _leaf(2, "0.75", "-1 0 0", "0 -1 0") +
                                  ["(Dynamics", "  m  =  3", "  r  =  0.5 0.5 0.5", "  v  =  0 0 1", ")Dynamics",
                                   ")Particle"]),
    "two dynamics sections": _j(_root(_leaf(1, "0.5", "1 2 3", "0 0 0") +
                                      ["(Particle", "(Dynamics", "  m = 2", ")Dynamics", "(Dynamics", "  m = 0.25",
                                       "  r = 0.125 0 0", ")Dynamics", ")Particle"])),
    "blank lines inside": _j(["(Particle", "", "  i = 4", "(Dynamics", "", "  m = 0.5", "", ")Dynamics", "",
                              ")Particle"] + [""] + ["(Particle", ")Particle"]),
    "crlf endings": _j(_root(_leaf(1, "0.3", "1 -2 3", "0.5 0 0") + _leaf(2, "0.7", "-1 2 -3", "0 0.5 0")), "\r\n"),
    "tabs": _j(["(Particle", "\ti\t=\t3", "(Dynamics", "\tm\t=\t1.5", "\tr\t=\t1\t2\t3", "\tv =\t-1 -2\t-3",
                ")Dynamics", ")Particle"]),
    "chapter inside dynamics": _j(["(Particle", "(Dynamics", "  m = 1", "(extra", "  m = 3", "  r = 1 1 1", ")extra",
                                   "  v = 2 2 2", ")Dynamics", ")Particle"]),
    "chapter in a particle body": _j(["(Particle", "(Foo", "  i = 7", "  name = foo7", ")Foo", "(Dynamics", "  m = 1",
                                      ")Dynamics", ")Particle"]),
    "particle-like chapters in log and star": _j(["(Particle", "(Log", "(Particle", "  m = 9", ")Particle", ")Log",
                                                  "(Star", "(Particle", "  m = 9", ")Particle", ")Star",
                                                  "(Hydro", "  r = 9 9 9", ")Hydro"] +
                                                 _leaf(5, "2", "0 0 1", "0 0 0") + [")Particle"]),
    "deep chain": _j(["(Particle"] * 1 + sum([["(Particle", "  i = %d" % k, "(Dynamics", "  m = %g" % (1 + k),
                                               "  r = %g 0 0" % (0.1 * k), ")Dynamics"] for k in range(12)], []) +
                     _leaf(99, "0.5", "0 0.25 0", "0 0 0.5") + [")Particle"] * 12 + [")Particle"]),
    "zero and negative parent mass": _j(_root(["(Particle"] + _leaf(1, "0", "1 0 0", "0 1 0") +
                                              _leaf(2, "0", "-1 0 0", "0 -1 0") + [")Particle", "(Particle"] +
                                              _leaf(3, "-1", "1 1 0", "0 0 0") + _leaf(4, "0.5", "0 1 1", "1 0 0") +
                                              [")Particle"])),
    "number forms": _j(_root(_leaf(1, "1.", ".5e1 -0 +7", "1e5 -1E-5 3.") +
                             _leaf(2, "   0.125   junk", "1 2 3 4", "-.5 +.25e+1 0x") +
                             _leaf(3, "4.9406564584124654e-324", "1e-320 2.2250738585072014e-308 1e300",
                                   "1.7976931348623157e308 -1e-310 0"))),
    "index and name forms": _j(_root(["(Particle", "  i = -5", "  name = a(b)c", "(Dynamics", "  m = 1", ")Dynamics",
                                      ")Particle", "(Particle", "  i = 99999999999", "  name =   spaced  name",
                                      ")Particle", "(Particle", "  i = +12abc", "  i = 13", ")Particle"])),
    "cut at 254 characters": _j(["(Particle", "(Dynamics", "  m  =  " + " " * 240 + "1.23456789",
                                 "  r  =  1 2 3" + " " * 300 + "4", "  v  =  0.5 0.25 " + " " * 230 + "0.125",
                                 ")Dynamics", ")Particle"]),
    "real_system_time and roots": _j(_root(_leaf(1, "1", "0 0 0", "0 0 0"), head=["(Dynamics", "  real_system_time = 2",
                                                                           "  system_time = 2.5", ")Dynamics"]) +
                                     ["(Particle", "(Dynamics", "  m = 3", ")Dynamics", ")Particle", "(Particle",
                                      ")Particle"]),
    "unterminated last line": _j(_root(_leaf(1, "1", "1 0 0", "0 0 0")))[:-1],
}


def random_valid_text(seed):
    """A random text the reference reads without error: random trees (the
    Dynamics section before or after the children), chapters in Log stories,
    Dynamics sections and particle bodies (holding key lines), repeated keys,
    blank lines inside particles, CRLF or LF, numbers in all strtod forms."""
    rng = np.random.default_rng(seed)
    nl = "\r\n" if rng.random() < 0.2 else "\n"
    out = []

    def num():
        x = float(rng.normal() * 10.0 ** rng.integers(-8, 8))
        return _num(rng, x) if rng.random() < 0.9 else rng.choice(["0", "-0", "1.", ".5", "+2e-3", "7E+01"])

    def dyn(keys=("m", "r", "v")):
        lines = ["(Dynamics"]
        for k in keys:
            if rng.random() < 0.85:
                lines.append("  %s  =  %s" % (k, num() if k == "m" else " ".join(num() for _ in range(3))))
        if rng.random() < 0.2:
            lines += ["(aside", "  m = %s" % num(), ")aside"]
        if rng.random() < 0.2:
            lines.append("  extra_key = 1 2 3")
        lines.append(")Dynamics")
        return lines

    def node(depth):
        lines = ["(Particle"]
        if rng.random() < 0.8:
            lines.append("  i = %d" % int(rng.integers(-5, 10 ** 6)))
        if rng.random() < 0.1:
            lines.append("  name = n%d" % int(rng.integers(0, 1000)))
        if rng.random() < 0.1:
            lines += ["(Note", "  i = %d" % int(rng.integers(0, 100)), ")Note"]
        if rng.random() < 0.1:
            lines.append("")
        lines += ["(Log"] + (["(ch", "  text", ")ch"] if rng.random() < 0.2 else []) + [")Log"]
        kids = int(rng.integers(2, 4)) if depth < 3 and rng.random() < 0.3 else 0
        after = rng.random() < 0.3
        if not after:
            lines += dyn()
        lines += ["(Hydro", ")Hydro", "(Star", ")Star"]
        for _ in range(kids):
            lines += node(depth + 1)
        if after:
            lines += dyn()
        lines.append(")Particle")
        return lines

    for r in range(int(rng.integers(1, 4))):
        root = ["(Particle", "(Log", ")Log"] + dyn(("m", "r", "v")) + (
            ["(Dynamics", "  system_time  =  %s" % num(), ")Dynamics"] if rng.random() < 0.7 else [])
        for _ in range(int(rng.integers(1, 12))):
            root += node(1)
        out += root + [")Particle"]
    return (nl.join(out) + nl).encode()
