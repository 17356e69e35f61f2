"""ctypes wrappers of the oracle libraries (test infrastructure only).

* ``G6Oracle``  -- oracle/_build/libg6oracle.so, the FP64 C restatement of
  the engine's semantics (oracle/g6_oracle.c).
* ``RefForce``  -- oracle/_ref/libref_force.so, Starlab's own FP64 path
  (predict_loworder + hdyn::flat_calculate_acc_and_jerk) built from the
  reference sources by oracle/build_ref.py.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libg6oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_force.so")

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
