"""The snapshot reader's oracle and boundary, on the CPU.

1. The C restatement of get_dyn (oracle/story_oracle.c) equals the
   reference's own reader (oracle/_ref/story_ref: get_dyn compiled from the
   reference sources) bit for bit on flat and hierarchical texts -- every
   node's parent, index, mass, position and velocity after
   check_and_correct_node, the leaves relative to their root, and the
   static system time -- and equals the committed golden vectors made by
   that reader (tests/golden/make_golden_story.py) where it is not built.
   The same on corner-case texts and seeded random structures, and
   format_story writes the bytes the reference's put_node writes.
2. With raw reading the values are exactly the written numbers.
3. Texts the reference cannot read give an error with a line number.
4. libg6b200.so exports every entry point include/g6b200_story.h declares,
   and without a GPU a reader cannot be created (no CPU path).
"""
import ctypes
import functools
import glob
import operator
import os
import re
import subprocess

import numpy as np
import pytest

from story_texts import MALFORMED, VARIANTS, flat_text, hierarchy_text, random_valid_text

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "story_*.npz")))


@pytest.fixture(scope="module")
def so():
    from oracle.oracle import StoryOracle
    return StoryOracle()


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype == np.float64:
        return np.array_equal(a.view(np.uint64), b.view(np.uint64))
    return np.array_equal(a, b)


FIELDS = ("parent", "index", "mass", "pos", "vel", "leaves_pos", "leaves_vel", "system_time")


def test_golden_present():
    assert len(GOLDEN) >= 2 + len(VARIANTS)


@pytest.mark.parametrize("path", GOLDEN, ids=os.path.basename)
def test_oracle_matches_golden(path, so):
    g = np.load(path)
    o = so.parse(g["text"].tobytes())
    for f in FIELDS:
        assert same(getattr(o, f), g[f]), f


@pytest.mark.parametrize("make", [lambda: flat_text(500, 21), lambda: hierarchy_text(4, roots=4, leaves_per_root=30),
                                  lambda: hierarchy_text(9, roots=1, leaves_per_root=300)],
                         ids=["flat500", "hier4x30", "hier1x300"])
def test_oracle_matches_reference_reader(make, so):
    from oracle.oracle import ref_story
    text = make()
    r = ref_story(text)
    if r is None:
        pytest.skip("oracle/_ref/story_ref not built (python oracle/build_ref.py)")
    o = so.parse(text)
    for f in FIELDS:
        assert same(getattr(o, f), getattr(r, f)), f
    named = [k for k, n in enumerate(r.names) if n is not None]
    assert [text[o.name_offset[k]:o.name_offset[k] + o.name_length[k]].decode() for k in named] == \
        [r.names[k] for k in named]


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_oracle_matches_reference_on_corner_cases(name, so):
    from oracle.oracle import ref_story
    text = VARIANTS[name]
    r = ref_story(text)
    if r is None:
        pytest.skip("oracle/_ref/story_ref not built (python oracle/build_ref.py)")
    o = so.parse(text)
    for f in FIELDS:
        assert same(getattr(o, f), getattr(r, f)), f
    got = [None if o.name_offset[k] < 0 else text[o.name_offset[k]:o.name_offset[k] + o.name_length[k]].decode()
           for k in range(o.parent.size)]
    assert got == r.names


def test_oracle_matches_reference_on_random_structures(so):
    from oracle.oracle import ref_story
    if ref_story(b"") is None:
        pytest.skip("oracle/_ref/story_ref not built (python oracle/build_ref.py)")
    for seed in range(60):
        text = random_valid_text(seed)
        r = ref_story(text)
        o = so.parse(text)
        for f in FIELDS:
            assert same(getattr(o, f), getattr(r, f)), (seed, f)


def test_format_story_writes_what_put_node_writes():
    """starlab_b200.story.format_story against the reference's own writer: a
    snapshot whose centre-of-mass sums are exact (equal masses, mirrored
    dyadic positions), so get_dyn moves nothing and put_node must give the
    same bytes back."""
    from oracle.oracle import ref_story_write
    from starlab_b200.story import format_story
    n = 16
    rng = np.random.default_rng(3)
    half = rng.integers(-64, 65, size=(n // 2, 3)) / 32.0
    x = np.concatenate([half, -half])
    v = np.concatenate([half[::-1] / 4, -half[::-1] / 4])
    text = format_story(np.full(n, 1.0 / n), x, v, log_lines=["  note = exact snapshot"])
    back = ref_story_write(text)
    if back is None:
        pytest.skip("oracle/_ref/story_ref not built (python oracle/build_ref.py)")
    assert back == text


def test_raw_values_are_the_written_numbers(so):
    text = flat_text(50, 2)
    o = so.parse(text, raw=True)
    rows = [l for l in text.decode().splitlines() if l.startswith("  r  =  ")]
    want = np.array([[float(t) for t in l.split()[2:5]] for l in rows])
    assert same(o.pos, want)
    c = so.parse(text)
    assert not same(c.pos[1:], o.pos[1:])   # the correction moved the leaves
    # the root's mass: its daughters' masses added one after another from 0
    # (functools.reduce; Python's sum() compensates rounding)
    assert c.mass[0] == functools.reduce(operator.add, o.mass[1:].tolist(), 0.0)


@pytest.mark.parametrize("name", sorted(MALFORMED))
def test_malformed_texts_are_errors(name, so):
    with pytest.raises(ValueError):
        so.parse(MALFORMED[name].encode())


def test_snapshots_end_at_an_empty_line(so):
    a = flat_text(10, 1)
    o = so.parse(a + b"\n" + b"garbage that is never read\n")
    assert o.parent.size == 11 and o.root_node.size == 1


def declared(header):
    text = re.sub(r"/\*.*?\*/", "", open(header).read(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(g6b200_story_[a-z_0-9]+)\s*\(", text,
                                 flags=re.M)))


def test_library_exports_the_story_abi():
    from starlab_b200 import LIB_PATH
    names = declared(os.path.join(REPO, "include", "g6b200_story.h"))
    assert len(names) >= 10, names
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], stdout=subprocess.PIPE, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert set(names) <= exported, set(names) - exported
    lib = ctypes.CDLL(LIB_PATH)
    assert all(hasattr(lib, n) for n in names)


def test_reader_fails_loudly_without_gpu():
    """No CPU path: without a device the reader cannot be created."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from starlab_b200.story import StoryError, StoryReader
    with pytest.raises(StoryError):
        StoryReader()
