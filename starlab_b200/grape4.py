"""Python binding of libh3b200.so (the B200 GRAPE-4 force engine).

Mirrors the GRAPE-4 (HARP-3) ABI that Starlab's ``hdyn_grape4.C`` drives
(``include/grape4.h:22-45``), with numpy arrays in place of pointers:

    h3 = H3Engine()                                        # h3open_
    h3.mjpdma_indirect(hostindex, x, v, aj, jj, m, t, 0)   # h3mjpdma_indirect_
    h3.mjpdma_start(0)                                     # h3mjpdma_start_
    h3.setti(ti)                                           # h3setti_
    h3.calc_firsthalf(nj, xi, vi, eps2, h2)                # h3calc_firsthalf_
    acc, jerk, pot = h3.calc_lasthalf(ni)                  # h3calc_lasthalf_
    h3.nbread(); h3.nblist(chip)                           # h3nbread_ / h3nblist_

``aj`` = acc/2 and ``jj`` = jerk/6 as kira stores them; ``eps2`` and ``h2``
are per i-slot and get the simulator's factor 2 inside the library.  Like
the reference simulator, the library reports misuse (ni above h3npipe_(),
an nj above h3jpmax_() in one DMA, an engine failure) by printing a message
and exiting the process.  There is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libh3b200.so")


class H3Stats(ctypes.Structure):
    _fields_ = [("calls", ctypes.c_longlong), ("slots", ctypes.c_longlong), ("computed", ctypes.c_longlong),
                ("interactions", ctypes.c_longlong), ("j_updates", ctypes.c_longlong),
                ("launches", ctypes.c_longlong)]


EXPORTS = ("h3open_", "h3close_", "h3npipe_", "h3setnboards_", "h3getnboards_", "h3wait_", "h3setti_",
           "h3setmode_", "h3setled_", "h3jpmax_", "h3jpdma_indirect_", "h3mjpdma_indirect_",
           "h3mjpdma_start_", "h3mjpdma_flush_", "h3calc_", "h3calc_firsthalf_", "h3calc_lasthalf_",
           "h3nbread_", "h3nblist_", "count_nblist_low", "h3setdebuglevel_", "h3checkdmabuffers_",
           "set_time_check_mode", "h3jpdma_flush_", "h3jpdma_reset_", "h3b200_last_error",
           "h3b200_get_stats")

_lib = None


def load_library(path=None):
    """Load (once) and return the ctypes handle of libh3b200.so."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError("libh3b200.so not built at %s (run python -m starlab_b200.build)" % p)
    lib = ctypes.CDLL(p)
    I, P = ctypes.c_int, ctypes.c_void_p
    IP = ctypes.POINTER(ctypes.c_int)
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "h3open_": (None, []), "h3close_": (None, []), "h3npipe_": (I, []),
        "h3setnboards_": (None, [IP]), "h3getnboards_": (I, []), "h3wait_": (ctypes.c_uint, []),
        "h3setti_": (None, [DP]), "h3jpmax_": (I, []),
        "h3jpdma_indirect_": (None, [IP, P, P, P, P, P, P, P, IP]),
        "h3mjpdma_indirect_": (None, [IP, P, P, P, P, P, P, P, IP, IP]),
        "h3mjpdma_start_": (None, [IP]), "h3mjpdma_flush_": (None, []),
        "h3calc_": (None, [IP, IP, P, P, P, P, P, P, P]),
        "h3calc_firsthalf_": (None, [IP, IP, P, P, P, P]),
        "h3calc_lasthalf_": (None, [IP, P, P, P]),
        "h3nbread_": (None, [IP]), "h3nblist_": (I, [IP, IP, P]), "count_nblist_low": (I, [I, I]),
        "h3b200_last_error": (ctypes.c_char_p, []),
        "h3b200_get_stats": (I, [ctypes.POINTER(H3Stats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _d(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _ip(v):
    return ctypes.byref(ctypes.c_int(int(v)))


class H3Engine:
    """The GRAPE-4 ABI of libh3b200.so (one global engine, like the hardware)."""

    def __init__(self, path=None):
        self.lib = load_library(path)
        self.lib.h3open_()

    def close(self):
        self.lib.h3close_()

    def npipe(self):
        return self.lib.h3npipe_()

    def jpmax(self):
        return self.lib.h3jpmax_()

    def setti(self, ti):
        self.lib.h3setti_(ctypes.byref(ctypes.c_double(float(ti))))

    def mjpdma_indirect(self, hostindex, x, v, aj, jj, m, t, buff_id=0):
        """h3mjpdma_indirect_: entry k is host element hostindex[k]-1 of the
        arrays and goes to j-address hostindex[k]-1."""
        hostindex = np.ascontiguousarray(hostindex, dtype=np.int32)
        n = x.shape[0]
        arrs = [_d(x, (n, 3)), _d(v, (n, 3)), _d(aj, (n, 3)), _d(jj, (n, 3)), _d(m, (n,)), _d(t, (n,))]
        self.lib.h3mjpdma_indirect_(_ip(hostindex.size), _p(hostindex), *[_p(a) for a in arrs], _ip(1),
                                    _ip(buff_id))

    def mjpdma_start(self, buff_id=0):
        self.lib.h3mjpdma_start_(_ip(buff_id))

    def mjpdma_flush(self):
        self.lib.h3mjpdma_flush_()

    def set_j_particles(self, x, v, aj, jj, m, t):
        """Every j-address 0..n-1 in one DMA (jpdma_nodes, hdyn_grape4.C:239-296)."""
        n = x.shape[0]
        self.mjpdma_indirect(np.arange(1, n + 1), x, v, aj, jj, m, np.broadcast_to(np.asarray(t, float), (n,)), 0)
        self.mjpdma_start(0)

    def calc_firsthalf(self, nj, xi, vi, eps2, h2):
        ni = xi.shape[0]
        self._hold = (_d(xi, (ni, 3)), _d(vi, (ni, 3)), _d(np.broadcast_to(np.asarray(eps2, float), (ni,))),
                      _d(np.broadcast_to(np.asarray(h2, float), (ni,))))
        self.lib.h3calc_firsthalf_(_ip(nj), _ip(ni), *[_p(a) for a in self._hold])

    def calc_lasthalf(self, ni):
        acc, jerk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
        self.lib.h3calc_lasthalf_(_ip(ni), _p(acc), _p(jerk), _p(pot))
        return acc, jerk, pot

    def calc(self, nj, xi, vi, eps2, h2):
        self.calc_firsthalf(nj, xi, vi, eps2, h2)
        return self.calc_lasthalf(xi.shape[0])

    def nbread(self):
        self.lib.h3nbread_(_ip(1))

    def nblist(self, chip, capacity=None):
        n = self.lib.count_nblist_low(0, int(chip))
        out = np.empty(max(n, 1) if capacity is None else capacity, dtype=np.int32)
        got = self.lib.h3nblist_(_ip(0), _ip(chip), _p(out))
        return out[:got].copy()

    def stats(self):
        s = H3Stats()
        self.lib.h3b200_get_stats(ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in H3Stats._fields_}
