"""Python binding of libg6b200.so (the B200 GRAPE-6 force engine).

Mirrors the g6 ABI that Starlab's ``hdyn_grape6.C`` drives
(``include/grape6.h:16-104``), with numpy arrays in place of pointers:

    eng = G6Engine(cluster_id=0, precision="mixed")
    eng.set_j_particles(address, tj, mass, k18, j6, a2, v, x)   # or set_j_particle
    eng.set_ti(ti)
    eng.calc_firsthalf(nj, index, xi, vi, eps2, h2)             # g6calc_firsthalf_
    acc, jerk, pot, nn = eng.calc_lasthalf2(ni)                 # g6calc_lasthalf2_
    eng.read_neighbour_list(); eng.get_neighbour_list(pipe)     # g6_*_neighbour_list_

Errors follow the reference's conventions (nonzero int returns) and are
raised here as ``G6Error`` carrying the code and the library's message.
There is no CPU fallback: without the built library or a GPU the calls
fail.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libg6b200.so")

FP64 = 0
MIXED = 1
_PREC = {"fp64": FP64, "mixed": MIXED, FP64: FP64, MIXED: MIXED}


class G6Error(RuntimeError):
    def __init__(self, what, code, msg):
        super().__init__("%s returned %d: %s" % (what, code, msg))
        self.code = code


class Stats(ctypes.Structure):
    _fields_ = [("calls", ctypes.c_longlong), ("interactions", ctypes.c_longlong),
                ("j_updates", ctypes.c_longlong), ("h2d_bytes", ctypes.c_longlong),
                ("d2h_bytes", ctypes.c_longlong), ("last_force_ms", ctypes.c_double),
                ("last_predict_ms", ctypes.c_double), ("last_call_ms", ctypes.c_double),
                ("launches", ctypes.c_longlong), ("refined", ctypes.c_longlong)]


_lib = None


def load_library(path=None):
    """Load (once) and return the ctypes handle of libg6b200.so."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError("libg6b200.so not built at %s (run python -m starlab_b200.build)" % p)
    lib = ctypes.CDLL(p)
    I, D, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    IP = ctypes.POINTER(ctypes.c_int)
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "g6_open_": (I, [IP]), "g6_close_": (I, [IP]), "g6_reset_": (I, [IP]),
        "g6_reset_fofpga_": (I, [IP]), "g6_npipes_": (I, []),
        "g6_open_special": (I, [I, IP]), "g6_open_special2": (I, [I, IP, I]),
        "g6_set_ti_": (None, [IP, DP]),
        "g6_set_j_particle_": (I, [IP, IP, IP, DP, DP, DP, P, P, P, P, P]),
        "g6calc_firsthalf_": (None, [IP, IP, IP, P, P, P, P, P, P, DP, P]),
        "g6calc_lasthalf_": (I, [IP, IP, IP, P, P, P, DP, P, P, P, P]),
        "g6calc_lasthalf2_": (I, [IP, IP, IP, P, P, P, DP, P, P, P, P, P]),
        "g6_read_neighbour_list_": (I, [IP]), "g6_read_neighbour_list_old_": (I, [IP]),
        "g6_get_neighbour_list_": (I, [IP, IP, IP, IP, P]),
        "g6_initialize_jp_buffer_": (I, [IP, IP]), "g6_flush_jp_buffer_": (I, [IP]),
        "g6_set_neighbour_list_sphere_": (None, [IP, DP]),
        "g6_set_tunit_": (None, [IP]), "g6_set_xunit_": (None, [IP]),
        "g6b200_set_precision": (I, [I, I]), "g6b200_get_precision": (I, [I]),
        "g6b200_set_npipes": (I, [I, I]), "g6b200_get_npipes": (I, [I]),
        "g6b200_set_config": (I, [I, I, I, I, I, I]), "g6b200_get_config": (I, [I, IP]),
        "g6b200_set_j_particles": (I, [I, I, P, P, P, P, P, P, P, P, P]),
        "g6b200_get_stats": (I, [I, ctypes.POINTER(Stats)]),
        "g6b200_sweep": (I, [I, I, I, I, D, P, P, P, P]),
        "g6b200_calc_pot": (I, [I, I, I, P, P, D, P]),
        "g6b200_energies": (I, [I, I, D, DP, DP, P]),
        "g6b200_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _vec(a, n):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != (n, 3):
        a = a.reshape(n, 3)
    return a


class G6Engine:
    """One engine instance (a GRAPE-6 ``cluster_id``)."""

    def __init__(self, cluster_id=0, precision=None, npipes=None, lib=None):
        self.lib = lib or load_library()
        self.cid = int(cluster_id)
        self._cid = ctypes.c_int(self.cid)
        if precision is not None:
            self.set_precision(precision)
        if npipes is not None:
            self.set_npipes(npipes)
        self._pending = None

    # -- lifecycle -----------------------------------------------------
    def _err(self, what, code):
        msg = self.lib.g6b200_last_error()
        raise G6Error(what, code, msg.decode() if msg else "")

    def open(self):
        rc = self.lib.g6_open_(ctypes.byref(self._cid))
        if rc:
            self._err("g6_open_", rc)

    def close(self):
        self.lib.g6_close_(ctypes.byref(self._cid))

    def reset(self):
        return self.lib.g6_reset_(ctypes.byref(self._cid))

    def npipes(self):
        return self.lib.g6b200_get_npipes(self.cid)

    def set_npipes(self, n):
        if self.lib.g6b200_set_npipes(self.cid, int(n)):
            raise ValueError("bad npipes %r" % n)

    def set_precision(self, p):
        if self.lib.g6b200_set_precision(self.cid, _PREC[p]):
            raise ValueError("bad precision %r" % p)

    def precision(self):
        return self.lib.g6b200_get_precision(self.cid)

    def set_config(self, il=0, r=1, warps=8, h=1, nsplit=1):
        if self.lib.g6b200_set_config(self.cid, il, r, warps, h, nsplit):
            raise ValueError("unsupported launch configuration")

    def last_config(self):
        out = (ctypes.c_int * 5)()
        self.lib.g6b200_get_config(self.cid, out)
        return tuple(out)

    def stats(self):
        s = Stats()
        self.lib.g6b200_get_stats(self.cid, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    # -- j-memory ------------------------------------------------------
    def set_j_particle(self, address, tj, mass, k18, j6, a2, v, x, index=None, dtj=1.0):
        """g6_set_j_particle_: one particle (vectors of length 3)."""
        a = ctypes.c_int(int(address))
        ix = ctypes.c_int(int(address if index is None else index))
        t, dt, m = ctypes.c_double(tj), ctypes.c_double(dtj), ctypes.c_double(mass)
        arrs = [np.ascontiguousarray(q, dtype=np.float64) for q in (k18, j6, a2, v, x)]
        rc = self.lib.g6_set_j_particle_(ctypes.byref(self._cid), ctypes.byref(a), ctypes.byref(ix),
                                         ctypes.byref(t), ctypes.byref(dt), ctypes.byref(m),
                                         *[_ptr(q) for q in arrs])
        if rc:
            self._err("g6_set_j_particle_", rc)

    def set_j_particles(self, tj, mass, j6, a2, v, x, k18=None, address=None, index=None):
        """Batched upload (g6b200_set_j_particles); vectors are (n, 3)."""
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        n = mass.shape[0]
        tj = np.ascontiguousarray(np.broadcast_to(np.asarray(tj, dtype=np.float64), (n,)))
        addr = None if address is None else np.ascontiguousarray(address, dtype=np.int32)
        idx = None if index is None else np.ascontiguousarray(index, dtype=np.int32)
        k = None if k18 is None else _vec(k18, n)
        arrs = [_vec(q, n) for q in (j6, a2, v, x)]
        rc = self.lib.g6b200_set_j_particles(self.cid, n, _ptr(addr), _ptr(idx), _ptr(tj), _ptr(mass),
                                             _ptr(k), *[_ptr(q) for q in arrs])
        if rc:
            self._err("g6b200_set_j_particles", rc)

    def flush(self):
        rc = self.lib.g6_flush_jp_buffer_(ctypes.byref(self._cid))
        if rc:
            self._err("g6_flush_jp_buffer_", rc)

    def set_ti(self, ti):
        t = ctypes.c_double(ti)
        self.lib.g6_set_ti_(ctypes.byref(self._cid), ctypes.byref(t))

    # -- force calls ---------------------------------------------------
    def calc_firsthalf(self, nj, index, xi, vi, eps2, h2=None, aold=None, j6old=None, phiold=None):
        index = np.ascontiguousarray(index, dtype=np.int32)
        ni = index.shape[0]
        xi, vi = _vec(xi, ni), _vec(vi, ni)
        hh = None if h2 is None else np.ascontiguousarray(np.broadcast_to(np.asarray(h2, np.float64), (ni,)))
        # aold/j6old/phiold are scaling hints the engine does not use: one
        # zero buffer, kept between calls
        if getattr(self, "_zeros3", None) is None or self._zeros3.shape[0] < max(ni, 1):
            self._zeros3, self._zeros1 = np.zeros((max(ni, 1), 3)), np.zeros(max(ni, 1))
        zeros3, zeros1 = self._zeros3, self._zeros1
        self._keep = (index, xi, vi, hh)
        c_nj, c_ni, c_e = ctypes.c_int(int(nj)), ctypes.c_int(ni), ctypes.c_double(eps2)
        self.lib.g6calc_firsthalf_(ctypes.byref(self._cid), ctypes.byref(c_nj), ctypes.byref(c_ni),
                                   _ptr(index), _ptr(xi), _ptr(vi),
                                   _ptr(zeros3 if aold is None else _vec(aold, ni)),
                                   _ptr(zeros3 if j6old is None else _vec(j6old, ni)),
                                   _ptr(zeros1 if phiold is None else np.ascontiguousarray(phiold, np.float64)),
                                   ctypes.byref(c_e), _ptr(hh))
        self._pending = (int(nj), ni, float(eps2))

    def calc_lasthalf2(self, ni=None, out=None):
        """g6calc_lasthalf2_; `out` = (acc, jerk, pot, nn) C-contiguous arrays
        to write into (else new ones are returned)."""
        nj, n, eps2 = self._pending
        ni = n if ni is None else ni
        if out is None:
            acc, jerk, pot, nn = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni), np.empty(ni, dtype=np.int32)
        else:
            acc, jerk, pot, nn = out
        index, xi, vi, hh = self._keep
        c_nj, c_ni, c_e = ctypes.c_int(nj), ctypes.c_int(ni), ctypes.c_double(eps2)
        rc = self.lib.g6calc_lasthalf2_(ctypes.byref(self._cid), ctypes.byref(c_nj), ctypes.byref(c_ni),
                                        _ptr(index), _ptr(xi), _ptr(vi), ctypes.byref(c_e), _ptr(hh),
                                        _ptr(acc), _ptr(jerk), _ptr(pot), _ptr(nn))
        if rc:
            self._err("g6calc_lasthalf2_", rc)
        return acc, jerk, pot, nn

    def calc_lasthalf(self, ni=None):
        nj, n, eps2 = self._pending
        ni = n if ni is None else ni
        acc = np.empty((ni, 3))
        jerk = np.empty((ni, 3))
        pot = np.empty(ni)
        index, xi, vi, hh = self._keep
        c_nj, c_ni, c_e = ctypes.c_int(nj), ctypes.c_int(ni), ctypes.c_double(eps2)
        rc = self.lib.g6calc_lasthalf_(ctypes.byref(self._cid), ctypes.byref(c_nj), ctypes.byref(c_ni),
                                       _ptr(index), _ptr(xi), _ptr(vi), ctypes.byref(c_e), _ptr(hh),
                                       _ptr(acc), _ptr(jerk), _ptr(pot))
        if rc:
            self._err("g6calc_lasthalf_", rc)
        return acc, jerk, pot

    def force(self, nj, index, xi, vi, eps2, h2=None):
        """firsthalf + lasthalf2 in one call, chunked by npipes."""
        index = np.ascontiguousarray(index, dtype=np.int32)
        ni = index.shape[0]
        xi, vi = _vec(xi, ni), _vec(vi, ni)
        npipes = self.npipes()
        outs = [np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni), np.empty(ni, dtype=np.int32)]
        for s in range(0, ni, npipes):
            e = min(ni, s + npipes)
            hh = None if h2 is None else np.broadcast_to(np.asarray(h2, np.float64), (ni,))[s:e]
            self.calc_firsthalf(nj, index[s:e], xi[s:e], vi[s:e], eps2, hh)
            self.calc_lasthalf2(out=tuple(o[s:e] for o in outs))
        return tuple(outs)

    def sweep(self, nj, i0=0, ni=None, eps2=0.0, copy_out=True):
        """Forces on the stored particles [i0, i0+ni) themselves
        (g6b200_sweep); returns (acc, jerk, pot, nn) or None when
        copy_out is False (results left in device memory)."""
        ni = nj - i0 if ni is None else ni
        if copy_out:
            acc, jerk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
            nn = np.empty(ni, dtype=np.int32)
            rc = self.lib.g6b200_sweep(self.cid, nj, i0, ni, eps2, _ptr(acc), _ptr(jerk), _ptr(pot), _ptr(nn))
        else:
            rc = self.lib.g6b200_sweep(self.cid, nj, i0, ni, eps2, None, None, None, None)
        if rc:
            self._err("g6b200_sweep", rc)
        return (acc, jerk, pot, nn) if copy_out else None

    def potential(self, nj, index, xi, eps2):
        """Potential only (g6b200_calc_pot), chunked by npipes: pot[ni] of
        the i-particles from the j-memory predicted to the current ti."""
        index = np.ascontiguousarray(index, dtype=np.int32)
        ni = index.shape[0]
        xi = _vec(xi, ni)
        pot = np.empty(ni)
        npipes = self.npipes()
        for s in range(0, ni, npipes):
            e = min(ni, s + npipes)
            rc = self.lib.g6b200_calc_pot(self.cid, int(nj), e - s, _ptr(index[s:e]),
                                          _ptr(np.ascontiguousarray(xi[s:e])), float(eps2), _ptr(pot[s:e]))
            if rc:
                self._err("g6b200_calc_pot", rc)
        return pot

    def energies(self, nj, eps2, want_pot=False):
        """g6b200_energies: (epot, ekin[, pot]) of the stored particles
        [0, nj) among themselves at the current ti."""
        ep, ek = ctypes.c_double(0), ctypes.c_double(0)
        pot = np.empty(nj) if want_pot else None
        rc = self.lib.g6b200_energies(self.cid, int(nj), float(eps2), ctypes.byref(ep), ctypes.byref(ek), _ptr(pot))
        if rc:
            self._err("g6b200_energies", rc)
        return (ep.value, ek.value, pot) if want_pot else (ep.value, ek.value)

    # -- neighbour lists -----------------------------------------------
    def read_neighbour_list(self):
        return self.lib.g6_read_neighbour_list_(ctypes.byref(self._cid))

    def get_neighbour_list(self, pipe, max_length=4096):
        nbl = np.empty(max(max_length, 1), dtype=np.int32)
        p, m, n = ctypes.c_int(pipe), ctypes.c_int(max_length), ctypes.c_int(0)
        rc = self.lib.g6_get_neighbour_list_(ctypes.byref(self._cid), ctypes.byref(p), ctypes.byref(m),
                                             ctypes.byref(n), _ptr(nbl))
        return rc, nbl[:min(n.value, max_length)].copy()
