"""ctypes loader of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module; the product path never does.  The oracle library is built by
oracle/Makefile from oracle/fosite_oracle.cpp.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from fosite_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libfosite_oracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_create.argtypes = [C.POINTER(abi.Config), C.POINTER(C.c_void_p)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_cell_count.argtypes = [C.c_void_p]
        L.orc_cell_count.restype = C.c_int64
        L.orc_vnum.argtypes = [C.c_void_p]
        L.orc_nfaces.argtypes = [C.c_void_p]
        L.orc_get_mesh.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_set_sound_speeds.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_set_state.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_first_step.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p]
        L.orc_compute_rhs.argtypes = [C.c_void_p]
        L.orc_calc_timestep.argtypes = [C.c_void_p]
        L.orc_calc_timestep.restype = C.c_double
        L.orc_get_status.argtypes = [C.c_void_p, C.POINTER(abi.Status)]
        L.orc_error.argtypes = [C.c_void_p]
        L.orc_error.restype = C.c_char_p
        L.orc_get_pointmass.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_set_fargo_velocity.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n=0):
    """Host threads of the oracle's data-parallel loops (n <= 0: keep the current count).

    Returns the number in use.  Results do not depend on it."""
    return int(lib().orc_set_threads(int(n)))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """Python handle on one oracle simulation (same config struct as the GPU library)."""

    def __init__(self, cfg):
        L = lib()
        h = C.c_void_p()
        rc = L.orc_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise RuntimeError("oracle create failed (%d)" % rc)
        self.h = h
        self.cfg = cfg
        self.nc = int(L.orc_cell_count(h))
        self.vnum = int(L.orc_vnum(h))
        self.nfaces = int(L.orc_nfaces(h))
        g = lambda n: 2 if n > 1 else 0
        self.shape = (cfg.knum + 2 * g(cfg.knum), cfg.jnum + 2 * g(cfg.jnum), cfg.inum + 2 * g(cfg.inum))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def mesh(self, which):
        out = np.zeros(self.nc)
        lib().orc_get_mesh(self.h, which, _ptr(out))
        return out.reshape(self.shape)

    def set_sound_speeds(self, bcc, fcs):
        bcc = np.ascontiguousarray(bcc, dtype=np.float64)
        fcs = np.ascontiguousarray(fcs, dtype=np.float64)
        lib().orc_set_sound_speeds(self.h, _ptr(bcc), _ptr(fcs))

    def set_state(self, which, data):
        data = np.ascontiguousarray(data, dtype=np.float64)
        assert data.size == self.nc * self.vnum
        lib().orc_set_state(self.h, which, _ptr(data))

    def get(self, which):
        n = self.nc if which == abi.BCCSOUND else self.nc * self.vnum
        out = np.zeros(n)
        lib().orc_get(self.h, which, _ptr(out))
        if which == abi.BCCSOUND:
            return out.reshape(self.shape)
        return out.reshape((self.vnum,) + self.shape)

    def first_step(self):
        return lib().orc_first_step(self.h)

    def step(self):
        return lib().orc_step(self.h)

    def compute_rhs(self):
        return lib().orc_compute_rhs(self.h)

    def calc_timestep(self):
        return lib().orc_calc_timestep(self.h)

    def status(self):
        st = abi.Status()
        lib().orc_get_status(self.h, C.byref(st))
        return st

    def set_fargo_velocity(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        rc = lib().orc_set_fargo_velocity(self.h, _ptr(w), w.size)
        if rc:
            raise RuntimeError("orc_set_fargo_velocity failed (%d)" % rc)

    def pointmass(self):
        """(mass, mdot) of the central point mass (accretion bookkeeping)."""
        m, d = C.c_double(), C.c_double()
        lib().orc_get_pointmass(self.h, C.byref(m), C.byref(d))
        return m.value, d.value
