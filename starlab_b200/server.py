"""Python binding of the force-call server (g6b200_srv_*).

    srv = Server(precision="mixed", hbm_budget=8 << 30)
    c = srv.open_cluster(n, eps2)                 # blocks until admitted
    srv.set_j(c, tj, mass, j6, a2, v, x)
    rid = srv.submit(c, ti, nj, index, xi, vi)    # any thread
    acc, jerk, pot, nn, latency_s = srv.wait(rid)
"""
import ctypes

import numpy as np

from .g6 import G6Error, load_library, _PREC


class SrvStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_longlong), ("requests", ctypes.c_longlong),
                ("interactions", ctypes.c_longlong), ("max_batch", ctypes.c_longlong), ("gpu_ms", ctypes.c_double),
                ("batch_ms", ctypes.c_double), ("queue_ms", ctypes.c_double)]


def _bind(lib):
    if getattr(lib, "_srv_bound", False):
        return
    P, I, D, L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    lib.g6b200_srv_create.restype = P
    lib.g6b200_srv_create.argtypes = [I, L, I, I]
    lib.g6b200_srv_open_cluster.argtypes = [P, L, D]
    lib.g6b200_srv_close_cluster.argtypes = [P, I]
    lib.g6b200_srv_set_j.argtypes = [P, I, I, P, P, P, P, P, P, P]
    lib.g6b200_srv_submit.restype = L
    lib.g6b200_srv_submit.argtypes = [P, I, D, I, I, P, P, P]
    lib.g6b200_srv_wait.argtypes = [P, L, P, P, P, P, ctypes.POINTER(ctypes.c_double)]
    lib.g6b200_srv_wait_batch.argtypes = [P, L, P, P, P, P, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
    lib.g6b200_srv_hold.argtypes = [P, I]
    lib.g6b200_srv_hold.restype = None
    lib.g6b200_srv_stats.argtypes = [P, ctypes.POINTER(SrvStats)]
    lib.g6b200_srv_destroy.argtypes = [P]
    lib.g6b200_srv_destroy.restype = None
    lib._srv_bound = True


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Server:
    def __init__(self, precision="mixed", hbm_budget=16 << 30, max_batch=1024, device=0):
        self.lib = load_library()
        _bind(self.lib)
        h = self.lib.g6b200_srv_create(int(device), int(hbm_budget), _PREC[precision], int(max_batch))
        if not h:
            raise G6Error("g6b200_srv_create", -1, self.lib.g6b200_last_error().decode())
        self.h = ctypes.c_void_p(h)

    def open_cluster(self, n_cap, eps2):
        c = self.lib.g6b200_srv_open_cluster(self.h, int(n_cap), float(eps2))
        if c < 0:
            raise G6Error("g6b200_srv_open_cluster", c, self.lib.g6b200_last_error().decode())
        return c

    def close_cluster(self, c):
        return self.lib.g6b200_srv_close_cluster(self.h, int(c))

    def set_j(self, c, tj, mass, j6, a2, v, x, address=None):
        mass = np.ascontiguousarray(mass, np.float64)
        n = mass.shape[0]
        tj = np.ascontiguousarray(np.broadcast_to(np.asarray(tj, np.float64), (n,)))
        arrs = [np.ascontiguousarray(q, np.float64).reshape(n, 3) for q in (j6, a2, v, x)]
        addr = None if address is None else np.ascontiguousarray(address, np.int32)
        rc = self.lib.g6b200_srv_set_j(self.h, int(c), n, _p(addr), _p(tj), _p(mass), *[_p(q) for q in arrs])
        if rc:
            raise G6Error("g6b200_srv_set_j", rc, self.lib.g6b200_last_error().decode())

    def submit(self, c, ti, nj, index, xi, vi):
        index = np.ascontiguousarray(index, np.int32)
        ni = index.shape[0]
        xi = np.ascontiguousarray(xi, np.float64).reshape(ni, 3)
        vi = np.ascontiguousarray(vi, np.float64).reshape(ni, 3)
        rid = self.lib.g6b200_srv_submit(self.h, int(c), float(ti), int(nj), ni, _p(index), _p(xi), _p(vi))
        if rid < 0:
            raise G6Error("g6b200_srv_submit", rid, "bad request")
        return rid, ni

    def wait(self, rid_ni):
        rid, ni = rid_ni
        acc, jerk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
        nn = np.empty(ni, dtype=np.int32)
        lat = ctypes.c_double(0)
        rc = self.lib.g6b200_srv_wait(self.h, rid, _p(acc), _p(jerk), _p(pot), _p(nn), ctypes.byref(lat))
        if rc:
            raise G6Error("g6b200_srv_wait", rc, self.lib.g6b200_last_error().decode())
        return acc, jerk, pot, nn, lat.value

    def wait_batch(self, rid_ni):
        """wait() plus (batch sequence number, calls in that batch)."""
        rid, ni = rid_ni
        acc, jerk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
        nn = np.empty(ni, dtype=np.int32)
        lat, b, bs = ctypes.c_double(0), ctypes.c_longlong(-1), ctypes.c_int(0)
        rc = self.lib.g6b200_srv_wait_batch(self.h, rid, _p(acc), _p(jerk), _p(pot), _p(nn), ctypes.byref(lat),
                                            ctypes.byref(b), ctypes.byref(bs))
        if rc:
            raise G6Error("g6b200_srv_wait_batch", rc, self.lib.g6b200_last_error().decode())
        return acc, jerk, pot, nn, lat.value, b.value, bs.value

    def hold(self, on=True):
        """Gather calls without dispatching them (released by hold(False))."""
        self.lib.g6b200_srv_hold(self.h, 1 if on else 0)

    def stats(self):
        st = SrvStats()
        self.lib.g6b200_srv_stats(self.h, ctypes.byref(st))
        return {k: getattr(st, k) for k, _ in SrvStats._fields_}

    def close(self):
        if self.h:
            self.lib.g6b200_srv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ResStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_longlong), ("calls", ctypes.c_longlong), ("launches", ctypes.c_longlong),
                ("recoveries", ctypes.c_longlong), ("max_batch", ctypes.c_int)]


def _bind_res(lib):
    if getattr(lib, "_res_bound", False):
        return
    P, I, D, L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    lib.g6b200_res_create.restype = P
    lib.g6b200_res_create.argtypes = [I, L, I, I]
    lib.g6b200_res_open_cluster.argtypes = [P, L, D]
    lib.g6b200_res_close_cluster.argtypes = [P, I]
    lib.g6b200_res_set_j.argtypes = [P, I, I, P, P, P, P, P, P, P]
    lib.g6b200_res_submit.restype = L
    lib.g6b200_res_submit.argtypes = [P, I, D, I, I, P, P, P]
    lib.g6b200_res_wait.argtypes = [P, L, P, P, P, P, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
    lib.g6b200_res_hold.argtypes = [P, I]
    lib.g6b200_res_hold.restype = None
    lib.g6b200_res_selftest_stall.argtypes = [P]
    lib.g6b200_res_selftest_stall.restype = None
    lib.g6b200_res_stats.argtypes = [P, ctypes.POINTER(ResStats)]
    lib.g6b200_res_destroy.argtypes = [P]
    lib.g6b200_res_destroy.restype = None
    lib._res_bound = True


class ResidentServer:
    """The device-resident serving loop (g6b200_res_*): the same calls as
    Server, served by one persistent kernel that polls a request ring in
    pinned host memory (no launch per call or per batch)."""

    def __init__(self, precision="mixed", hbm_budget=16 << 30, max_batch=1024, device=0):
        self.lib = load_library()
        _bind_res(self.lib)
        h = self.lib.g6b200_res_create(int(device), int(hbm_budget), _PREC[precision], int(max_batch))
        if not h:
            raise G6Error("g6b200_res_create", -1, self.lib.g6b200_last_error().decode())
        self.h = ctypes.c_void_p(h)

    def open_cluster(self, n_cap, eps2):
        c = self.lib.g6b200_res_open_cluster(self.h, int(n_cap), float(eps2))
        if c < 0:
            raise G6Error("g6b200_res_open_cluster", c, self.lib.g6b200_last_error().decode())
        return c

    def close_cluster(self, c):
        return self.lib.g6b200_res_close_cluster(self.h, int(c))

    def set_j(self, c, tj, mass, j6, a2, v, x, address=None):
        mass = np.ascontiguousarray(mass, np.float64)
        n = mass.shape[0]
        tj = np.ascontiguousarray(np.broadcast_to(np.asarray(tj, np.float64), (n,)))
        arrs = [np.ascontiguousarray(q, np.float64).reshape(n, 3) for q in (j6, a2, v, x)]
        addr = None if address is None else np.ascontiguousarray(address, np.int32)
        rc = self.lib.g6b200_res_set_j(self.h, int(c), n, _p(addr), _p(tj), _p(mass), *[_p(q) for q in arrs])
        if rc:
            raise G6Error("g6b200_res_set_j", rc, self.lib.g6b200_last_error().decode())

    def submit(self, c, ti, nj, index, xi, vi):
        index = np.ascontiguousarray(index, np.int32)
        ni = index.shape[0]
        xi = np.ascontiguousarray(xi, np.float64).reshape(ni, 3)
        vi = np.ascontiguousarray(vi, np.float64).reshape(ni, 3)
        rid = self.lib.g6b200_res_submit(self.h, int(c), float(ti), int(nj), ni, _p(index), _p(xi), _p(vi))
        if rid < 0:
            raise G6Error("g6b200_res_submit", rid, self.lib.g6b200_last_error().decode())
        return rid, ni

    def wait_batch(self, rid_ni):
        """(acc, jerk, pot, nn, latency_s, batch sequence number, calls in that batch)."""
        rid, ni = rid_ni
        acc, jerk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
        nn = np.empty(ni, dtype=np.int32)
        lat, b, bs = ctypes.c_double(0), ctypes.c_longlong(-1), ctypes.c_int(0)
        rc = self.lib.g6b200_res_wait(self.h, rid, _p(acc), _p(jerk), _p(pot), _p(nn), ctypes.byref(lat),
                                      ctypes.byref(b), ctypes.byref(bs))
        if rc:
            raise G6Error("g6b200_res_wait", rc, self.lib.g6b200_last_error().decode())
        return acc, jerk, pot, nn, lat.value, b.value, bs.value

    def wait(self, rid_ni):
        return self.wait_batch(rid_ni)[:5]

    def hold(self, on=True):
        self.lib.g6b200_res_hold(self.h, 1 if on else 0)

    def selftest_stall(self):
        self.lib.g6b200_res_selftest_stall(self.h)

    def stats(self):
        st = ResStats()
        self.lib.g6b200_res_stats(self.h, ctypes.byref(st))
        d = {k: getattr(st, k) for k, _ in ResStats._fields_}
        d["requests"] = d["calls"]
        return d

    def close(self):
        if self.h:
            self.lib.g6b200_res_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
