"""Python host mirror of the fosite time-step interface, driving the C ABI.

``Simulation`` follows the sequence of fosite's own driver (fosite.f90:
Setup -> InitData -> FirstStep -> Step/Run) with the state kept on the GPU:
``set_state`` stands for InitData's Timedisc%pvar/cvar fill, ``first_step`` for
fosite%FirstStep, ``step``/``run`` for fosite%Step/Run, and ``get`` for reading
Timedisc%cvar/pvar back.  Every call goes through include/fosite_gpu.h; there
is no CPU path: if the CUDA library is missing the import fails.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def lib_path(exact=False):
    name = "libfosite_gpu_exact.so" if exact else "libfosite_gpu.so"
    return os.path.join(_HERE, "lib", name)


def lib(exact=False):
    """Load the CUDA library; raise if it was not built (no fallback exists)."""
    if exact in _libs:
        return _libs[exact]
    path = lib_path(exact)
    if not os.path.exists(path):
        raise RuntimeError("fosite_b200: CUDA library %s is missing; run fosite_b200/build.py" % path)
    L = C.CDLL(path)
    L.fgpu_config_init.argtypes = [C.POINTER(abi.Config)]
    L.fgpu_create.argtypes = [C.POINTER(abi.Config), C.c_int, C.POINTER(C.c_void_p)]
    L.fgpu_destroy.argtypes = [C.c_void_p]
    L.fgpu_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
    L.fgpu_state_size.argtypes = [C.c_void_p]
    L.fgpu_state_size.restype = C.c_int64
    L.fgpu_cell_count.argtypes = [C.c_void_p]
    L.fgpu_cell_count.restype = C.c_int64
    L.fgpu_vnum.argtypes = [C.c_void_p]
    L.fgpu_get_mesh.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
    L.fgpu_set_sound_speeds.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]
    L.fgpu_upload_state.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
    L.fgpu_download.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
    L.fgpu_first_step.argtypes = [C.c_void_p]
    L.fgpu_step.argtypes = [C.c_void_p]
    L.fgpu_run.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    L.fgpu_compute_rhs.argtypes = [C.c_void_p]
    L.fgpu_calc_timestep.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.fgpu_set_output_time.argtypes = [C.c_void_p, C.c_double]
    L.fgpu_get_status.argtypes = [C.c_void_p, C.POINTER(abi.Status)]
    L.fgpu_synchronize.argtypes = [C.c_void_p]
    L.fgpu_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.fgpu_set_profiling.argtypes = [C.c_void_p, C.c_int]
    L.fgpu_get_stats.argtypes = [C.c_void_p, C.POINTER(abi.Stats)]
    L.fgpu_reset_stats.argtypes = [C.c_void_p]
    L.fgpu_autotune.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.fgpu_stage_layout.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.fgpu_get_pointmass.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.fgpu_set_fargo_velocity.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    L.fgpu_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
    L.fgpu_batch_destroy.argtypes = [C.c_void_p]
    L.fgpu_batch_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
    L.fgpu_batch_size.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.fgpu_batch_run.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_int)]
    L.fgpu_batch_autotune.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.fgpu_batch_layout.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.fgpu_measure_l2_read.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.fgpu_batch_enqueue.argtypes = [C.c_void_p, C.c_int64]
    L.fgpu_batch_collect.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    _libs[exact] = L
    return L


def l2_read_gbs(device=0, mb=16, passes=512):
    """Measured read bandwidth (GB/s) of an L2-resident array of mb MB (fgpu_measure_l2_read)."""
    v = C.c_double(0.0)
    rc = lib().fgpu_measure_l2_read(int(device), int(mb), int(passes), C.byref(v))
    if rc != 0:
        raise FositeError(rc, "fgpu_measure_l2_read failed")
    return float(v.value)


class FositeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("fosite_b200 error %d: %s" % (code, msg))
        self.code = code


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Simulation:
    """One grid, one CUDA stream, state resident in HBM."""

    def __init__(self, cfg, device=-1, exact=False):
        self.L = lib(exact)
        self.cfg = abi.finalize_config(abi.config_copy(cfg))
        h = C.c_void_p()
        rc = self.L.fgpu_create(C.byref(self.cfg), device, C.byref(h))
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.L.fgpu_last_error(None, buf, 512)
            raise FositeError(rc, buf.value.decode())
        self.h = h
        self.vnum = int(self.L.fgpu_vnum(h))
        self.ncells = int(self.L.fgpu_cell_count(h))
        g = lambda n: 2 if n > 1 else 0
        c = self.cfg
        self.shape = (c.knum + 2 * g(c.knum), c.jnum + 2 * g(c.jnum), c.inum + 2 * g(c.inum))
        self.nfaces = 2 * sum(1 for n in (c.inum, c.jnum, c.knum) if n > 1)

    def close(self):
        if getattr(self, "h", None):
            self.L.fgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, soft_ok=True):
        if rc < 0 or (rc > 0 and not soft_ok):
            buf = C.create_string_buffer(512)
            self.L.fgpu_last_error(self.h, buf, 512)
            raise FositeError(rc, buf.value.decode())
        return rc

    # ---- mesh / physics data
    def mesh(self, which):
        out = np.zeros(self.ncells)
        self._check(self.L.fgpu_get_mesh(self.h, which, _ptr(out), out.size))
        return out.reshape(self.shape)

    def set_sound_speeds(self, bccsound, fcsound):
        b = np.ascontiguousarray(bccsound, dtype=np.float64)
        f = np.ascontiguousarray(fcsound, dtype=np.float64)
        self._check(self.L.fgpu_set_sound_speeds(self.h, _ptr(b), b.size, _ptr(f), f.size))

    # ---- state
    def set_state(self, which, data):
        d = np.ascontiguousarray(data, dtype=np.float64)
        self._check(self.L.fgpu_upload_state(self.h, which, _ptr(d), d.size))

    def get(self, which):
        n = self.ncells if which == abi.BCCSOUND else self.ncells * self.vnum
        out = np.zeros(n)
        self._check(self.L.fgpu_download(self.h, which, _ptr(out), out.size))
        if which == abi.BCCSOUND:
            return out.reshape(self.shape)
        return out.reshape((self.vnum,) + self.shape)

    # ---- stepping
    def first_step(self):
        return self._check(self.L.fgpu_first_step(self.h))

    def step(self):
        return self._check(self.L.fgpu_step(self.h))

    def run(self, n):
        done = C.c_int64(0)
        rc = self._check(self.L.fgpu_run(self.h, int(n), C.byref(done)))
        return rc, int(done.value)

    def compute_rhs(self):
        self._check(self.L.fgpu_compute_rhs(self.h))
        return self.get(abi.RHS)

    def calc_timestep(self):
        d = C.c_double()
        self._check(self.L.fgpu_calc_timestep(self.h, C.byref(d)))
        return d.value

    def fluxes(self, which):
        """Interface fluxes of the last compute_rhs (abi.XFLUX, YFLUX or ZFLUX), ghost-padded like
        fosite's Fluxes%xfluxdydz: index i holds the flux through the face between cells i and i+1."""
        return self.get(which)

    def set_output_time(self, tout):
        """The next output time; step() clips dt so that a step ends there."""
        self._check(self.L.fgpu_set_output_time(self.h, float(tout)))

    def status(self):
        st = abi.Status()
        self._check(self.L.fgpu_get_status(self.h, C.byref(st)))
        return st

    def set_fargo_velocity(self, w):
        """Background velocity of FARGO type 2: one value per padded i (inum+4) for transport
        along y, per padded j (jnum+4) along x."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        self._check(self.L.fgpu_set_fargo_velocity(self.h, _ptr(w), w.size))

    def pointmass(self):
        """(mass, mdot) of the central point mass; changes only with accretion."""
        m, d = C.c_double(), C.c_double()
        self._check(self.L.fgpu_get_pointmass(self.h, C.byref(m), C.byref(d)))
        return m.value, d.value

    def synchronize(self):
        self._check(self.L.fgpu_synchronize(self.h))

    def set_stream(self, stream_handle):
        """Enqueue on a caller stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self.L.fgpu_set_stream(self.h, C.c_void_p(stream_handle or None)))

    def set_profiling(self, on):
        self._check(self.L.fgpu_set_profiling(self.h, 1 if on else 0))

    def stats(self):
        st = abi.Stats()
        self._check(self.L.fgpu_get_stats(self.h, C.byref(st)))
        return st

    def reset_stats(self):
        self._check(self.L.fgpu_reset_stats(self.h))

    def autotune(self, reps=3):
        """Time every stage-kernel layout on this grid and keep the fastest; returns its id."""
        v = C.c_int(0)
        self._check(self.L.fgpu_autotune(self.h, int(reps), C.byref(v)))
        return int(v.value)

    def stage_layout(self):
        """(layout id, z chunk) of the stage kernel later steps launch."""
        v, k = C.c_int(0), C.c_int(0)
        self._check(self.L.fgpu_stage_layout(self.h, C.byref(v), C.byref(k)))
        return int(v.value), int(k.value)


class Batch:
    """Ensemble of Simulations advanced together by batched persistent launches.

    The members must have run ``first_step``; they stay usable (status, get)
    and must outlive the batch.  Stepping a member on its own while it belongs
    to a live batch is not allowed.
    """

    def __init__(self, sims):
        if not sims:
            raise ValueError("empty batch")
        self.sims = list(sims)
        self.L = self.sims[0].L
        arr = (C.c_void_p * len(self.sims))(*[s.h for s in self.sims])
        b = C.c_void_p()
        rc = self.L.fgpu_batch_create(arr, len(self.sims), C.byref(b))
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.L.fgpu_batch_last_error(None, buf, 512)
            raise FositeError(rc, buf.value.decode())
        self.b = b
        m, t = C.c_int(0), C.c_int(0)
        self.L.fgpu_batch_size(b, C.byref(m), C.byref(t))
        self.tiles = int(t.value)

    def _check(self, rc):
        if rc < 0:
            buf = C.create_string_buffer(512)
            self.L.fgpu_batch_last_error(self.b, buf, 512)
            raise FositeError(rc, buf.value.decode())
        return rc

    def run(self, n):
        """Advance every member by n steps; returns how many are still running."""
        a = C.c_int(0)
        self._check(self.L.fgpu_batch_run(self.b, int(n), C.byref(a)))
        return int(a.value)

    def enqueue(self, n):
        """Queue n steps of every member without waiting (see collect)."""
        self._check(self.L.fgpu_batch_enqueue(self.b, int(n)))

    def collect(self):
        """Wait for the queued steps; returns how many members are still running."""
        a = C.c_int(0)
        self._check(self.L.fgpu_batch_collect(self.b, C.byref(a)))
        return int(a.value)

    def autotune(self, reps=3):
        v = C.c_int(0)
        self._check(self.L.fgpu_batch_autotune(self.b, int(reps), C.byref(v)))
        return int(v.value)

    def layout(self):
        """The batch's stage layout (0/2/3 shared-memory tiles, 6 TMA-staged tiles)."""
        v = C.c_int(0)
        self._check(self.L.fgpu_batch_layout(self.b, C.byref(v)))
        return int(v.value)

    def close(self):
        if getattr(self, "b", None):
            self.L.fgpu_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
