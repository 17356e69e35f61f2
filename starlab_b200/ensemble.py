"""Python binding of the ensemble integrator (g6b200_ens_*).

    ens = Ensemble([m0, m1, ...], [x0, x1, ...], [v0, v1, ...], eps2=[...], eta=0.02, precision="mixed")
    ens.start()
    stats = ens.run(1.0)                 # batched: one merged launch per iteration
    stats = ens.run(1.0, per_cluster=True)  # plain engine, one call per cluster per block
    ek, ep = ens.energies()
"""
import ctypes

import numpy as np

from .g6 import G6Error, load_library, _PREC


class EnsStats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("interactions", ctypes.c_longlong),
                ("iterations", ctypes.c_longlong), ("launches", ctypes.c_longlong), ("tuned_h", ctypes.c_int),
                ("tuned_tasks", ctypes.c_int), ("lane_interactions", ctypes.c_longlong)]


def _bind(lib):
    if getattr(lib, "_ens_bound", False):
        return
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.g6b200_ens_create.restype = P
    lib.g6b200_ens_create.argtypes = [I, P, P, D, I, I]
    lib.g6b200_ens_set_cluster.argtypes = [P, I, P, P, P]
    lib.g6b200_ens_start.argtypes = [P]
    lib.g6b200_ens_run.argtypes = [P, D, I, I, ctypes.POINTER(EnsStats)]
    lib.g6b200_ens_energies.argtypes = [P, P]
    lib.g6b200_ens_get_cluster.argtypes = [P, I, P, P, P, P, P, P, P]
    lib.g6b200_ens_destroy.argtypes = [P]
    lib.g6b200_ens_destroy.restype = None
    lib._ens_bound = True


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Ensemble:
    def __init__(self, masses, positions, velocities, eps2, eta=0.02, precision="mixed", device=0):
        self.lib = load_library()
        _bind(self.lib)
        self.n = np.array([len(m) for m in masses], dtype=np.int32)
        self.eps2 = np.ascontiguousarray(np.broadcast_to(np.asarray(eps2, np.float64), (len(masses),)))
        h = self.lib.g6b200_ens_create(len(masses), _p(self.n), _p(self.eps2), float(eta), _PREC[precision],
                                       int(device))
        if not h:
            raise G6Error("g6b200_ens_create", -1, self.lib.g6b200_last_error().decode())
        self.h = ctypes.c_void_p(h)
        for c, (m, x, v) in enumerate(zip(masses, positions, velocities)):
            m = np.ascontiguousarray(m, np.float64)
            x = np.ascontiguousarray(x, np.float64)
            v = np.ascontiguousarray(v, np.float64)
            self._chk("g6b200_ens_set_cluster", self.lib.g6b200_ens_set_cluster(self.h, c, _p(m), _p(x), _p(v)))

    def _chk(self, what, rc):
        if rc:
            raise G6Error(what, rc, self.lib.g6b200_last_error().decode())

    def start(self):
        self._chk("g6b200_ens_start", self.lib.g6b200_ens_start(self.h))

    def run(self, t_end, per_cluster=False, tune=False):
        st = EnsStats()
        self._chk("g6b200_ens_run", self.lib.g6b200_ens_run(self.h, float(t_end), int(per_cluster), int(tune),
                                                            ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in EnsStats._fields_}

    def energies(self):
        out = np.empty(2 * len(self.n))
        self._chk("g6b200_ens_energies", self.lib.g6b200_ens_energies(self.h, _p(out)))
        return out[0::2].copy(), out[1::2].copy()

    def get(self, c):
        """dict with m, x, v, acc, jerk, t, dt of cluster c."""
        n = int(self.n[c])
        out = dict(m=np.empty(n), x=np.empty((n, 3)), v=np.empty((n, 3)), acc=np.empty((n, 3)),
                   jerk=np.empty((n, 3)), t=np.empty(n), dt=np.empty(n))
        self._chk("g6b200_ens_get_cluster", self.lib.g6b200_ens_get_cluster(
            self.h, c, *[_p(out[k]) for k in ("m", "x", "v", "acc", "jerk", "t", "dt")]))
        return out

    def close(self):
        if self.h:
            self.lib.g6b200_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
