"""ctypes wrappers of the oracle libraries (test infrastructure only).

* ``G6Oracle``  -- oracle/_build/libg6oracle.so, the FP64 C restatement of
  the engine's semantics (oracle/g6_oracle.c).
* ``RefForce``  -- oracle/_ref/libref_force.so, Starlab's own FP64 path
  (predict_loworder + hdyn::flat_calculate_acc_and_jerk) built from the
  reference sources by oracle/build_ref.py.
* ``G4Oracle``  -- oracle/_build/libg4oracle.so, the FP64 C restatement of
  the GRAPE-4 pipeline (oracle/g4_oracle.c).
* ``Harp3Sim``  -- oracle/_ref/libharp3sim.so, the reference's own IEEE
  GRAPE-4 simulator (src/harpsims/harp3fastsim.c) driven through its ABI.
* ``StoryOracle`` -- oracle/_build/libstoryoracle.so, the sequential C
  restatement of the reference's snapshot reader (oracle/story_oracle.c).
* ``ref_story`` -- oracle/_ref/story_ref, the reference's own get_dyn run on
  a text, every value printed exactly.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libg6oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_force.so")
G4_ORACLE_LIB = os.path.join(HERE, "_build", "libg4oracle.so")
HARP3_LIB = os.path.join(HERE, "_ref", "libharp3sim.so")
STORY_ORACLE_LIB = os.path.join(HERE, "_build", "libstoryoracle.so")
STORY_REF = os.path.join(HERE, "_ref", "story_ref")

_P = ctypes.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


class G6Oracle:
    def __init__(self, path=ORACLE_LIB):
        if not os.path.exists(path):
            raise ImportError("oracle library missing: %s" % path)
        self.lib = ctypes.CDLL(path)
        I, D = ctypes.c_int, ctypes.c_double
        self.lib.g6o_predict.argtypes = [I, D, _P, _P, _P, _P, _P, _P, _P]
        self.lib.g6o_force.argtypes = [I, _P, _P, _P, _P, I, _P, _P, _P, D, _P, _P, _P, _P, _P]
        self.lib.g6o_neighbours.argtypes = [I, _P, _P, I, _P, _P, _P, I, _P, _P, _P]

    def predict(self, ti, tj, x, v, a2, j6):
        n = x.shape[0]
        tj = _c(np.broadcast_to(np.asarray(tj, np.float64), (n,)))
        xp, vp = np.empty((n, 3)), np.empty((n, 3))
        self.lib.g6o_predict(n, float(ti), _p(tj), _p(_c(x)), _p(_c(v)), _p(_c(a2)), _p(_c(j6)), _p(xp), _p(vp))
        return xp, vp

    def force(self, xj, vj, mj, index_i, xi, vi, eps2, jindex=None):
        nj = xj.shape[0]
        jindex = _c(np.arange(nj) if jindex is None else jindex, np.int32)
        index_i = _c(index_i, np.int32)
        ni = index_i.shape[0]
        acc, jerk = np.empty((ni, 3)), np.empty((ni, 3))
        pot, nn_r2 = np.empty(ni), np.empty(ni)
        nn = np.empty(ni, dtype=np.int32)
        self.lib.g6o_force(nj, _p(_c(xj)), _p(_c(vj)), _p(_c(mj)), _p(jindex), ni, _p(index_i),
                           _p(_c(xi)), _p(_c(vi)), float(eps2), _p(acc), _p(jerk), _p(pot), _p(nn), _p(nn_r2))
        return acc, jerk, pot, nn, nn_r2

    def neighbours(self, xj, index_i, xi, h2, include_self=True, jindex=None):
        """Return a list of ascending int arrays, one per i."""
        nj = xj.shape[0]
        jindex = _c(np.arange(nj) if jindex is None else jindex, np.int32)
        index_i = _c(index_i, np.int32)
        ni = index_i.shape[0]
        h2 = _c(np.broadcast_to(np.asarray(h2, np.float64), (ni,)))
        ln = np.empty(ni, dtype=np.int32)
        off = np.empty(ni + 1, dtype=np.int64)
        args = (nj, _p(_c(xj)), _p(jindex), ni, _p(index_i), _p(_c(xi)), _p(h2), int(include_self), _p(ln), _p(off))
        self.lib.g6o_neighbours(*args, None)
        out = np.empty(int(off[ni]), dtype=np.int32)
        self.lib.g6o_neighbours(*args, _p(out))
        return [out[off[i]:off[i + 1]] for i in range(ni)]


class RefForce:
    """Starlab's FP64 CPU force path on a flat tree (kira -0)."""

    def __init__(self, path=REF_LIB):
        if not os.path.exists(path):
            raise ImportError("reference oracle not built: %s (python oracle/build_ref.py)" % path)
        self.lib = ctypes.CDLL(path)
        I, D = ctypes.c_int, ctypes.c_double
        self.lib.ref_flat_force.restype = I
        self.lib.ref_flat_force.argtypes = [I, _P, _P, _P, _P, _P, _P, D, D, I, _P,
                                            _P, _P, _P, _P, _P, _P, _P, _P, I, _P]

    def force(self, mass, pos, vel, acc, jerk, tj, ti, eps, ilist=None, nthreads=1, want_pred=False):
        n = mass.shape[0]
        ilist = _c(np.arange(n) if ilist is None else ilist, np.int32)
        ni = ilist.shape[0]
        tj = _c(np.broadcast_to(np.asarray(tj, np.float64), (n,)))
        a_o, j_o = np.empty((ni, 3)), np.empty((ni, 3))
        p_o, d_o = np.empty(ni), np.empty(ni)
        nn_o = np.empty(ni, dtype=np.int32)
        pp = np.empty((n, 3)) if want_pred else None
        pv = np.empty((n, 3)) if want_pred else None
        eps2 = ctypes.c_double(0)
        secs = ctypes.c_double(0)
        rc = self.lib.ref_flat_force(n, _p(_c(mass)), _p(_c(pos)), _p(_c(vel)), _p(_c(acc)), _p(_c(jerk)),
                                     _p(tj), float(ti), float(eps), ni, _p(ilist), _p(a_o), _p(j_o), _p(p_o),
                                     _p(nn_o), _p(d_o), _p(pp), _p(pv), ctypes.byref(eps2), int(nthreads),
                                     ctypes.byref(secs))
        if rc:
            raise RuntimeError("ref_flat_force failed: %d" % rc)
        out = dict(acc=a_o, jerk=j_o, pot=p_o, nn=nn_o, dnn_sq=d_o, eps2=eps2.value, seconds=secs.value)
        if want_pred:
            out["pred_pos"], out["pred_vel"] = pp, pv
        return out


class G4Oracle:
    """GRAPE-4 pipeline restated in C (predictor and pair loop of
    harp3fastsim.c, plus the potential the simulator leaves at 0)."""

    def __init__(self, path=G4_ORACLE_LIB):
        if not os.path.exists(path):
            raise ImportError("oracle library missing: %s" % path)
        self.lib = ctypes.CDLL(path)
        I, D = ctypes.c_int, ctypes.c_double
        self.lib.g4o_predict.argtypes = [I, D, _P, _P, _P, _P, _P, _P, _P]
        self.lib.g4o_force.argtypes = [I, _P, _P, _P, I, _P, _P, _P, _P, _P, _P, _P, _P, _P, I]

    def predict(self, ti, tj, x, v, aj, jj):
        n = x.shape[0]
        tj = _c(np.broadcast_to(np.asarray(tj, np.float64), (n,)))
        xp, vp = np.empty((n, 3)), np.empty((n, 3))
        self.lib.g4o_predict(n, float(ti), _p(tj), _p(_c(x)), _p(_c(v)), _p(_c(aj)), _p(_c(jj)), _p(xp), _p(vp))
        return xp, vp

    def force(self, xj, vj, mj, xi, vi, eps2, h2, nbcap=None):
        """acc, jerk, pot and the neighbour lists (ascending) per i-slot."""
        nj, ni = xj.shape[0], xi.shape[0]
        eps2 = _c(np.broadcast_to(np.asarray(eps2, np.float64), (ni,)))
        h2 = _c(np.broadcast_to(np.asarray(h2, np.float64), (ni,)))
        acc, jerk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
        cnt = np.empty(ni, dtype=np.int32)
        cap = nj if nbcap is None else nbcap
        lists = np.empty((ni, max(cap, 1)), dtype=np.int32)
        self.lib.g4o_force(nj, _p(_c(xj)), _p(_c(vj)), _p(_c(mj)), ni, _p(_c(xi)), _p(_c(vi)), _p(eps2), _p(h2),
                           _p(acc), _p(jerk), _p(pot), _p(cnt), _p(lists), cap)
        nb = [lists[i, :min(cnt[i], cap)].copy() for i in range(ni)]
        return acc, jerk, pot, cnt, nb


class Harp3Sim:
    """The reference's GRAPE-4 simulator through its own ABI.

    Its static limits (harp3fastsim.c:23-26, 31): 1000 j-particles, 3 i per
    call, 26 j per DMA buffer, 1024 neighbours per i (unchecked: keep lists
    shorter).  It returns pot = 0 (:281).
    """
    NMAX, IPMAX, JPMAX, NNBMAX = 1000, 3, 26, 1024

    def __init__(self, path=HARP3_LIB):
        if not os.path.exists(path):
            raise ImportError("reference GRAPE-4 simulator not built: %s (python oracle/build_ref.py)" % path)
        self.lib = ctypes.CDLL(path)
        self.lib.h3nblist_.restype = ctypes.c_int

    def _i(self, v):
        return ctypes.byref(ctypes.c_int(int(v)))

    def load(self, x, v, aj, jj, m, t):
        n = x.shape[0]
        assert n <= self.NMAX
        x, v, aj, jj = _c(x), _c(v), _c(aj), _c(jj)
        m = _c(m)
        t = _c(np.broadcast_to(np.asarray(t, np.float64), (n,)))
        for b0 in range(0, n, self.JPMAX):
            idx = _c(np.arange(b0 + 1, min(b0 + self.JPMAX, n) + 1), np.int32)
            self.lib.h3mjpdma_indirect_(self._i(idx.size), _p(idx), _p(x), _p(v), _p(aj), _p(jj), _p(m), _p(t),
                                        self._i(1), self._i(0))
            self.lib.h3mjpdma_start_(self._i(0))

    def force(self, ti, nj, xi, vi, eps2, h2):
        """acc, jerk and neighbour lists for every i (3 per call)."""
        ni = xi.shape[0]
        eps2 = _c(np.broadcast_to(np.asarray(eps2, np.float64), (ni,)))
        h2 = _c(np.broadcast_to(np.asarray(h2, np.float64), (ni,)))
        xi, vi = _c(xi), _c(vi)
        self.lib.h3setti_(ctypes.byref(ctypes.c_double(float(ti))))
        acc, jerk = np.empty((ni, 3)), np.empty((ni, 3))
        lists = []
        buf = np.empty(self.NNBMAX, dtype=np.int32)
        for i0 in range(0, ni, self.IPMAX):
            k = min(self.IPMAX, ni - i0)
            a, jk, p = np.empty((k, 3)), np.empty((k, 3)), np.empty(k)
            self.lib.h3calc_firsthalf_(self._i(nj), self._i(k), _p(_c(xi[i0:i0 + k])), _p(_c(vi[i0:i0 + k])),
                                       _p(_c(eps2[i0:i0 + k])), _p(_c(h2[i0:i0 + k])))
            self.lib.h3calc_lasthalf_(self._i(k), _p(a), _p(jk), _p(p))
            acc[i0:i0 + k], jerk[i0:i0 + k] = a, jk
            for c in range(k):
                got = self.lib.h3nblist_(self._i(0), self._i(c), _p(buf))
                lists.append(buf[:got].copy())
        return acc, jerk, lists


class StorySnapshot:
    """Flat arrays of a parse (same names as starlab_b200.story.Snapshot)."""


def leaves_relative_to_root(parent, pos, vel):
    """Leaves (nodes without daughters, roots excluded) in pre-order, with
    positions/velocities summed from the leaf up to the root (excluded),
    starting at +0 -- something_relative_to_root, dyn_tt.C:94-110."""
    n = parent.size
    has_d = np.zeros(n, bool)
    has_d[parent[parent >= 0]] = True
    leaves = np.flatnonzero((~has_d) & (parent >= 0)).astype(np.int32)
    x = np.zeros((leaves.size, 3))
    v = np.zeros((leaves.size, 3))
    cur = leaves.copy()
    while True:
        act = parent[cur] >= 0
        if not act.any():
            break
        x[act] = x[act] + pos[cur[act]]
        v[act] = v[act] + vel[cur[act]]
        cur = np.where(act, parent[cur], cur)
    return leaves, x, v


class StoryOracle:
    """The C restatement of get_dyn over a whole text."""

    def __init__(self, path=STORY_ORACLE_LIB):
        if not os.path.exists(path):
            raise ImportError("story oracle library missing: %s" % path)
        self.lib = ctypes.CDLL(path)
        LLP = ctypes.POINTER(ctypes.c_longlong)
        self.lib.so_parse.restype = ctypes.c_void_p
        self.lib.so_parse.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_int, LLP, LLP, LLP,
                                      ctypes.POINTER(ctypes.c_char_p)]
        self.lib.so_error.argtypes = [ctypes.c_void_p]
        self.lib.so_get.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 9
        self.lib.so_free.argtypes = [ctypes.c_void_p]

    def parse(self, text, raw=False):
        """A StorySnapshot, or raises ValueError(line, what) on an error."""
        nn, nr, el = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        what = ctypes.c_char_p()
        h = self.lib.so_parse(text, len(text), 1 if raw else 0, ctypes.byref(nn), ctypes.byref(nr), ctypes.byref(el),
                              ctypes.byref(what))
        try:
            if self.lib.so_error(h):
                raise ValueError(int(el.value), what.value.decode() if what.value else "")
            n, r = nn.value, nr.value
            s = StorySnapshot()
            s.parent, s.index = np.empty(n, np.int32), np.empty(n, np.int32)
            s.name_offset, s.name_length = np.empty(n, np.int32), np.empty(n, np.int32)
            s.mass, s.pos, s.vel = np.empty(n), np.empty((n, 3)), np.empty((n, 3))
            s.root_node, s.system_time = np.empty(r, np.int32), np.empty(r)
            self.lib.so_get(h, _p(s.parent), _p(s.index), _p(s.name_offset), _p(s.name_length), _p(s.mass),
                            _p(s.pos), _p(s.vel), _p(s.root_node), _p(s.system_time))
        finally:
            self.lib.so_free(h)
        s.leaves_node, s.leaves_pos, s.leaves_vel = leaves_relative_to_root(s.parent, s.pos, s.vel)
        s.leaves_mass = s.mass[s.leaves_node]
        s.leaves_index = s.index[s.leaves_node]
        return s


def ref_story(text, path=STORY_REF, timeout=600):
    """Run the reference's get_dyn on text (oracle/_ref/story_ref): a
    StorySnapshot with names as strings, or None if the harness is not
    built.  A reference exit shows as RuntimeError."""
    import subprocess
    if not os.path.exists(path):
        return None
    r = subprocess.run([path], input=text, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference reader exited %d: %s" % (r.returncode, r.stderr[-500:].decode("latin-1")))
    parent, index, names, vals, lv, times = [], [], [], [], [], []
    for line in r.stdout.decode("latin-1").splitlines():
        f = line.split(" ")
        if f[0] == "P":
            parent.append(int(f[1]))
            index.append(int(f[2]))
            ln, _, nm = f[3].partition(":")
            names.append(None if int(ln) < 0 else nm)
            vals.append([float.fromhex(x) for x in f[4:11]])
        elif f[0] == "L":
            lv.append([float.fromhex(x) for x in f[1:7]])
        elif f[0] == "T":
            times.append(float.fromhex(f[1]))
    s = StorySnapshot()
    s.parent = np.array(parent, np.int32)
    s.index = np.array(index, np.int32)
    s.names = names
    v = np.array(vals, np.float64).reshape(-1, 7)
    s.mass, s.pos, s.vel = v[:, 0].copy(), v[:, 1:4].copy(), v[:, 4:7].copy()
    l6 = np.array(lv, np.float64).reshape(-1, 6)
    s.leaves_pos, s.leaves_vel = l6[:, :3].copy(), l6[:, 3:].copy()
    s.system_time = np.array(times)
    return s


def ref_story_write(text, path=STORY_REF, timeout=600):
    """The reference's get_dyn + put_node on text (story_ref -w): the text
    the reference writes back, or None if the harness is not built."""
    import subprocess
    if not os.path.exists(path):
        return None
    r = subprocess.run([path, "-w"], input=text, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference reader exited %d" % r.returncode)
    return r.stdout


def ref_story_seconds(path_to_text, path=STORY_REF, timeout=900):
    """Seconds the reference's get_dyn loop takes on a file (story_ref -t)."""
    import subprocess
    with open(path_to_text, "rb") as f:
        r = subprocess.run([path, "-t"], stdin=f, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference reader exited %d" % r.returncode)
    return float(r.stdout.split()[1])
