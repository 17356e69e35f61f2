"""Starlab story-format snapshots on the GPU: Python binding of the reader in
libg6b200.so (``include/g6b200_story.h``) and a writer of the same format.

The reader stands in for the reference's ``get_dyn`` loop
(``src/node/dyn/util/dyn_io.C:280-296``): every snapshot in a text is parsed
on the device, bit for bit as the reference reads it, and returned as flat
arrays::

    rd = StoryReader()
    snap = rd.parse(open("cluster.snap", "rb").read())
    snap.leaves_mass, snap.leaves_pos, snap.leaves_vel     # j-particles, root frame
    snap.parent, snap.mass, snap.pos, snap.vel            # every node, pre-order

``raw=True`` keeps the values as written (no ``check_and_correct_node``).
Errors raise ``StoryError`` with the line number.  There is no CPU path:
without the built library or a GPU the calls fail.

``format_story`` writes a flat snapshot (a root and n leaves) laid out as
the reference's ``put_node`` writes one (``src/node/util/tree_io.C:412+``;
the root's Star section with the unset scale factors,
``src/node/util/starbase_io.C:56-79``), numbers with "%.18g" as
``put_real_number`` / ``put_real_vector`` (``src/std/util_io.C:215-360``) at
the default precision; the root's Log holds the given lines.
"""
import ctypes

import numpy as np

from .g6 import load_library

RAW = 1


class StoryError(RuntimeError):
    pass


class Info(ctypes.Structure):
    _fields_ = [("bytes", ctypes.c_longlong), ("lines", ctypes.c_longlong), ("n_nodes", ctypes.c_longlong),
                ("n_leaves", ctypes.c_longlong), ("n_roots", ctypes.c_longlong), ("max_depth", ctypes.c_int)]


def _bind(lib):
    if getattr(lib, "_story_bound", False):
        return lib
    P, I, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    sig = {
        "g6b200_story_create": (P, [I]),
        "g6b200_story_destroy": (None, [P]),
        "g6b200_story_error": (ctypes.c_char_p, [P]),
        "g6b200_story_parse": (I, [P, P, LL, I, ctypes.POINTER(Info)]),
        "g6b200_story_parse_device": (I, [P, P, LL, I, ctypes.POINTER(Info)]),
        "g6b200_story_nodes": (I, [P, P, P, P, P, P]),
        "g6b200_story_names": (I, [P, P, P]),
        "g6b200_story_leaves": (I, [P, P, P, P, P, P]),
        "g6b200_story_roots": (I, [P, P, P]),
        "g6b200_story_device_leaves": (I, [P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    lib._story_bound = True
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Snapshot:
    """Arrays of one parse: nodes (pre-order over all snapshots), leaves
    (relative to their root), roots."""

    def __init__(self, info, text=None):
        self.info = info
        self.text = text

    def name(self, node):
        off, n = int(self.name_offset[node]), int(self.name_length[node])
        if off < 0 or self.text is None:
            return None
        return bytes(self.text[off:off + n]).decode("latin-1")


class StoryReader:
    def __init__(self, device=0, lib=None):
        self.lib = _bind(lib or load_library())
        self.h = self.lib.g6b200_story_create(int(device))
        if not self.h:
            raise StoryError("g6b200_story_create failed on device %d" % device)

    def close(self):
        if self.h:
            self.lib.g6b200_story_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise StoryError("%s returned %d: %s" % (what, rc, self.lib.g6b200_story_error(self.h).decode()))

    def parse_info(self, text, raw=False):
        """Parse host bytes; only the summary (the arrays stay on the device)."""
        buf = text if isinstance(text, bytes) else bytes(text)
        info = Info()
        self._check(self.lib.g6b200_story_parse(self.h, buf, len(buf), RAW if raw else 0, ctypes.byref(info)),
                    "g6b200_story_parse")
        return info

    def parse_device(self, ptr, nbytes, raw=False):
        """Parse text already in device memory (16-byte aligned pointer)."""
        info = Info()
        self._check(self.lib.g6b200_story_parse_device(self.h, ctypes.c_void_p(int(ptr)), int(nbytes),
                                                       RAW if raw else 0, ctypes.byref(info)),
                    "g6b200_story_parse_device")
        return info

    def parse(self, text, raw=False):
        """Parse host bytes and copy every result array back."""
        info = self.parse_info(text, raw)
        return self.fetch(info, text)

    def fetch(self, info, text=None):
        s = Snapshot(info, text)
        n, nl, nr = info.n_nodes, info.n_leaves, info.n_roots
        s.parent = np.empty(n, np.int32)
        s.index = np.empty(n, np.int32)
        s.mass = np.empty(n)
        s.pos = np.empty((n, 3))
        s.vel = np.empty((n, 3))
        self._check(self.lib.g6b200_story_nodes(self.h, _p(s.parent), _p(s.index), _p(s.mass), _p(s.pos), _p(s.vel)),
                    "g6b200_story_nodes")
        s.name_offset = np.empty(n, np.int64)
        s.name_length = np.empty(n, np.int32)
        self._check(self.lib.g6b200_story_names(self.h, _p(s.name_offset), _p(s.name_length)), "g6b200_story_names")
        s.leaves_node = np.empty(nl, np.int32)
        s.leaves_index = np.empty(nl, np.int32)
        s.leaves_mass = np.empty(nl)
        s.leaves_pos = np.empty((nl, 3))
        s.leaves_vel = np.empty((nl, 3))
        self._check(self.lib.g6b200_story_leaves(self.h, _p(s.leaves_node), _p(s.leaves_index), _p(s.leaves_mass),
                                                 _p(s.leaves_pos), _p(s.leaves_vel)), "g6b200_story_leaves")
        s.root_node = np.empty(nr, np.int32)
        s.system_time = np.empty(nr)
        self._check(self.lib.g6b200_story_roots(self.h, _p(s.root_node), _p(s.system_time)), "g6b200_story_roots")
        return s

    def device_leaves(self):
        """Device addresses of the last parse's leaf arrays (mass[n], pos[n][3],
        vel[n][3]), valid until the next parse: for device-side consumers."""
        m, x, v = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self.lib.g6b200_story_device_leaves(self.h, ctypes.byref(m), ctypes.byref(x), ctypes.byref(v)),
                    "g6b200_story_device_leaves")
        return m.value, x.value, v.value

    def leaves(self, info):
        """Leaves only (mass, pos, vel), the arrays a force engine loads."""
        nl = info.n_leaves
        m, x, v = np.empty(nl), np.empty((nl, 3)), np.empty((nl, 3))
        self._check(self.lib.g6b200_story_leaves(self.h, None, None, _p(m), _p(x), _p(v)), "g6b200_story_leaves")
        return m, x, v


def _g(x):
    return "%.18g" % x


def format_story(mass, pos, vel, index=None, system_time=0.0, log_lines=(), root_pos=(0.0, 0.0, 0.0)):
    """Story text of a flat snapshot: a root holding len(mass) leaves."""
    mass = np.asarray(mass, np.float64)
    pos = np.asarray(pos, np.float64)
    vel = np.asarray(vel, np.float64)
    n = mass.size
    idx = np.arange(1, n + 1) if index is None else np.asarray(index)
    out = ["(Particle", "  N = %d" % n, "(Log"]
    out += list(log_lines)
    out += [")Log", "(Dynamics", "  system_time  =  " + _g(system_time), "  m  =  " + _g(mass.sum()),
            "  r  =  %s %s %s" % tuple(_g(c) for c in root_pos), "  v  =  0 0 0", ")Dynamics", "(Hydro", ")Hydro",
            "(Star", "  mass_scale     =  -1", "  size_scale     =  -1", "  time_scale     =  -1", ")Star"]
    ms = [_g(x) for x in mass.tolist()]
    ps = [" ".join(_g(c) for c in row) for row in pos.tolist()]
    vs = [" ".join(_g(c) for c in row) for row in vel.tolist()]
    for k in range(n):
        out += ["(Particle", "  i = %d" % int(idx[k]), "  N = 1", "(Log", ")Log", "(Dynamics", "  m  =  " + ms[k],
                "  r  =  " + ps[k], "  v  =  " + vs[k], ")Dynamics", "(Hydro", ")Hydro", "(Star", ")Star",
                ")Particle"]
    out.append(")Particle")
    return ("\n".join(out) + "\n").encode()
