"""The story-format snapshot reader on the GPU, through the C ABI
(include/g6b200_story.h), against the oracle (oracle/story_oracle.c, itself
pinned to the reference's get_dyn): bit for bit on every node and leaf,
after check_and_correct_node and raw; text from host memory and already on
the device; the reader reused across texts of different sizes; inputs the
reference cannot read and forms this reader does not convert rejected with a
line number; a 262144-body snapshot.
"""
import numpy as np
import pytest

from story_texts import MALFORMED, VARIANTS, flat_text, hierarchy_text

pytestmark = pytest.mark.gpu

FIELDS = ("parent", "index", "mass", "pos", "vel", "leaves_pos", "leaves_vel", "leaves_mass", "system_time")


@pytest.fixture(scope="module")
def rd():
    from starlab_b200.story import StoryReader
    r = StoryReader()
    yield r
    r.close()


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


def check(g, o):
    for f in FIELDS:
        assert same(getattr(g, f), getattr(o, f)), f
    assert same(g.name_offset, o.name_offset) and same(g.name_length, o.name_length)
    assert same(g.root_node, o.root_node)
    assert same(g.leaves_node, o.leaves_node)


TEXTS = {
    "flat1000": lambda: flat_text(1000, 31),
    "hier_seed1": lambda: hierarchy_text(1),
    "hier_seed2_5roots": lambda: hierarchy_text(2, roots=5, leaves_per_root=25),
    "hier_seed3_deep": lambda: hierarchy_text(3, roots=1, leaves_per_root=400),
}


@pytest.mark.parametrize("name", sorted(TEXTS))
@pytest.mark.parametrize("raw", [False, True])
def test_matches_oracle(name, raw, rd, so):
    text = TEXTS[name]()
    check(rd.parse(text, raw=raw), so.parse(text, raw=raw))


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_corner_cases_match_oracle(name, rd, so):
    text = VARIANTS[name]
    check(rd.parse(text), so.parse(text))
    check(rd.parse(text, raw=True), so.parse(text, raw=True))


def test_matches_golden(rd):
    import glob
    import os
    for path in sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "story_*.npz"))):
        g = np.load(path)
        s = rd.parse(g["text"].tobytes())
        for f in ("parent", "index", "mass", "pos", "vel", "leaves_pos", "leaves_vel", "system_time"):
            assert same(getattr(s, f), g[f]), (path, f)


def test_text_on_device(rd, so):
    import torch
    text = hierarchy_text(5, roots=2, leaves_per_root=50)
    d = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    info = rd.parse_device(d.data_ptr(), d.numel())
    check(rd.fetch(info, text), so.parse(text))


def test_reuse_across_sizes(rd, so):
    for n in (3000, 10, 700, 0):
        text = flat_text(n, 40 + n) if n else b""
        g = rd.parse(text)
        if n == 0:
            assert g.info.n_nodes == 0
            continue
        check(g, so.parse(text))


def test_end_of_list_and_unterminated_line(rd, so):
    a = flat_text(20, 1)
    for text in (a + b"\n" + b"never read (\n", a[:-1], a + b"trailing words"):
        check(rd.parse(text), so.parse(text))


@pytest.mark.parametrize("name", sorted(MALFORMED))
def test_malformed_is_an_error(name, rd):
    from starlab_b200.story import StoryError
    with pytest.raises(StoryError, match="line"):
        rd.parse(MALFORMED[name].encode())


@pytest.mark.parametrize("text", [
    b"(Particle\n  (Dynamics\n  m = 2\n)Dynamics\n)Particle\n",            # indented section line
    b"(Particle\n(Dynamics\n(Dummy\n)Dummy\n)Dynamics\n)Particle\n",        # chapter named like its section
    b"(Particle\n(Dynamics\n  m = 0x1p3\n)Dynamics\n)Particle\n",          # hexadecimal float
], ids=["indented", "conflict", "hex"])
def test_unsupported_forms_are_errors(text, rd):
    from starlab_b200.story import StoryError
    with pytest.raises(StoryError):
        rd.parse(text)


def test_large_snapshot(rd, so):
    text = flat_text(262144, 77)
    g = rd.parse(text)
    o = so.parse(text)
    assert g.info.n_leaves == 262144
    for f in ("leaves_mass", "leaves_pos", "leaves_vel", "mass", "parent"):
        assert same(getattr(g, f), getattr(o, f)), f


def test_text_above_2gb(rd, so):
    """Byte offsets past 2^31: 2.2 GB of Log lines ahead of the particles."""
    head = flat_text(1000, 9)
    k = head.index(b"(Log\n") + len(b"(Log\n")
    filler = (b"  " + b"a" * 100 + b"\n") * 21_400_000
    text = head[:k] + filler + head[k:]
    del filler
    assert len(text) > 2 ** 31 + 2 ** 25  # particle lines beyond byte 2^31
    g = rd.parse(text)
    o = so.parse(text)
    assert g.info.n_leaves == 1000 and g.info.bytes == len(text)
    for f in ("leaves_mass", "leaves_pos", "leaves_vel", "mass", "pos", "parent", "index", "system_time"):
        assert same(getattr(g, f), getattr(o, f)), f


def test_device_leaves_are_the_copied_ones(rd):
    from cuda.bindings import runtime as rt
    text = flat_text(3000, 12)
    info = rd.parse_info(text)
    m, x, v = rd.leaves(info)
    pm, px, pv = rd.device_leaves()
    for host, ptr in ((m, pm), (x, px), (v, pv)):
        got = np.empty_like(host)
        (e,) = rt.cudaMemcpy(got.ctypes.data, ptr, got.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert e == rt.cudaError_t.cudaSuccess
        assert same(got, host)
