"""fosite's self-describing binary output format, for GPU results and restarts.

Format (io/fileio_binary.f90:30-50, WriteHeader :215-247, WriteKey :298-362,
WriteNode :398-575), little endian, 8-byte reals, 4-byte integers:

  header  "FOSITE" + "II" + chr(0) + "%2d%2d" % (realsize, intsize)   13 bytes
  record  [key length][key][type][byte count][dims...][data]

Types follow common/common_dict.f90:93-105 (1 int, 2 real, 6/7/8/12 real
arrays of 2/3/4/5 dimensions).  Array records carry 3 dimensions, or 4/5 when
those extents exceed 1; the byte count includes the dimension integers.  Keys
are the paths of fosite's IO dictionary ("/timedisc/density", "/mesh/bary_curv",
"/config/mesh/inum", ...), data in Fortran order (i fastest).

`write_state` writes the primitive state (Timedisc%pvar interior, the names of
Physics%pvarname), the time and the mesh bary centres, with the configuration
values that describe them; `read` parses any file of this format;
`restart_config` / `restart_state` turn a file back into a config with its
start time and a ghost-padded pvar for `Simulation.set_state` (the pattern of
examples/restart.f90:49-170).
"""
import struct

import numpy as np

from . import abi

DICT_INT, DICT_REAL, DICT_CHAR, DICT_BOOL = 1, 2, 3, 4
DICT_REAL_ONED, DICT_REAL_TWOD, DICT_REAL_THREED, DICT_REAL_FOURD = 5, 6, 7, 8
DICT_INT_ONED, DICT_REAL_FIVED = 9, 12
_ARRAY_TYPES = (DICT_REAL_TWOD, DICT_REAL_THREED, DICT_REAL_FOURD, DICT_REAL_FIVED)

HEADER = b"FOSITE" + b"II" + b"\x00" + b" 8 4"
REALSIZE, INTSIZE = 8, 4


def pvar_names(cfg):
    """Physics%pvarname in variable order (physics_euler.f90:165-203)."""
    nd = sum(1 for n in (cfg.inum, cfg.jnum, cfg.knum) if n > 1)
    names = ["density"] + ["xvelocity", "yvelocity", "zvelocity"][:nd]
    if cfg.physics == abi.EULER:
        names.append("pressure")
    return names


class _Writer:
    def __init__(self, f):
        self.f = f
        f.write(HEADER)

    def _key(self, key, typ, nbytes, dims=None):
        k = key.encode("ascii")
        d = [] if dims is None else list(dims)
        self.f.write(struct.pack("<i", len(k)) + k + struct.pack("<ii", typ, nbytes + INTSIZE * len(d)))
        if d:
            self.f.write(struct.pack("<%di" % len(d), *d))

    def scalar(self, key, value):
        if isinstance(value, (int, np.integer)):
            self._key(key, DICT_INT, INTSIZE)
            self.f.write(struct.pack("<i", int(value)))
        else:
            self._key(key, DICT_REAL, REALSIZE)
            self.f.write(struct.pack("<d", float(value)))

    def array(self, key, a):
        """a: numpy array indexed [..., k, j, i] (C order); written i fastest."""
        a = np.ascontiguousarray(a, dtype="<f8")
        fdims = list(a.shape[::-1])                       # Fortran extents (i, j, k, ...)
        while len(fdims) < 3:
            fdims.append(1)
        typ = {2: DICT_REAL_TWOD, 3: DICT_REAL_THREED, 4: DICT_REAL_FOURD, 5: DICT_REAL_FIVED}[max(3, a.ndim)]
        n = 3                                              # WriteKey: 4th/5th extent only if > 1
        if len(fdims) > 3 and fdims[3] > 1:
            n = 4
        if len(fdims) > 4 and fdims[4] > 1:
            n = 5
        self._key(key, typ, a.size * REALSIZE, fdims[:n])
        self.f.write(a.tobytes(order="C"))


def write_state(path, cfg, time, pvar, bary=None):
    """Write a ghost-padded primitive state ([V, KG, JG, IG], fosite's pvar) and its time."""
    cfg_items = [("/config/mesh/geometry", int(cfg.geometry)), ("/config/mesh/inum", int(cfg.inum)),
                 ("/config/mesh/jnum", int(cfg.jnum)), ("/config/mesh/knum", int(cfg.knum)),
                 ("/config/mesh/xmin", cfg.xmin), ("/config/mesh/xmax", cfg.xmax),
                 ("/config/mesh/ymin", cfg.ymin), ("/config/mesh/ymax", cfg.ymax),
                 ("/config/mesh/zmin", cfg.zmin), ("/config/mesh/zmax", cfg.zmax),
                 ("/config/mesh/gparam", cfg.gparam), ("/config/physics/problem", int(cfg.physics)),
                 ("/config/physics/gamma", cfg.gamma), ("/config/physics/cs", cfg.csiso),
                 ("/config/timedisc/stoptime", cfg.stoptime)]
    sl = [slice(None)]
    for n in (cfg.knum, cfg.jnum, cfg.inum):
        sl.append(slice(2, -2) if n > 1 else slice(None))
    interior = np.asarray(pvar)[tuple(sl)]
    with open(path, "wb") as f:
        w = _Writer(f)
        for k, v in cfg_items:
            w.scalar(k, v)
        if bary is not None:
            w.array("/mesh/bary_curv", bary)
        w.scalar("/timedisc/time", float(time))
        for name, a in zip(pvar_names(cfg), interior):
            w.array("/timedisc/" + name, a)


def read(path):
    """Parse a file into {key: value}; arrays come back indexed [..., k, j, i]."""
    out = {}
    with open(path, "rb") as f:
        head = f.read(13)
        if head[:6] != b"FOSITE" or head[6:8] != b"II":
            raise ValueError("not a little-endian fosite binary file")
        rsize, isize = int(head[9:11]), int(head[11:13])
        if (rsize, isize) != (REALSIZE, INTSIZE):
            raise ValueError("unsupported real/int sizes %d/%d" % (rsize, isize))
        while True:
            b = f.read(4)
            if len(b) < 4:
                break
            (klen,) = struct.unpack("<i", b)
            key = f.read(klen).decode("ascii")
            typ, nbytes = struct.unpack("<ii", f.read(8))
            if typ in _ARRAY_TYPES:
                dims = list(struct.unpack("<3i", f.read(12)))
                # 4/5 dimensions are present only when their extents exceed 1
                while int(np.prod(dims)) * REALSIZE + INTSIZE * len(dims) < nbytes:
                    dims.append(struct.unpack("<i", f.read(4))[0])
                data = np.frombuffer(f.read(int(np.prod(dims)) * REALSIZE), dtype="<f8")
                out[key] = data.reshape(dims[::-1]).copy()
            elif typ == DICT_INT:
                out[key] = struct.unpack("<i", f.read(nbytes))[0]
            elif typ == DICT_REAL:
                out[key] = struct.unpack("<d", f.read(nbytes))[0]
            else:
                out[key] = f.read(nbytes)
    return out


def restart_config(cfg, data):
    """A copy of cfg that starts at the file's time (starttime, timedisc_base.f90:295)."""
    c = abi.config_copy(cfg)
    c.starttime = float(data["/timedisc/time"])
    return c


def restart_state(cfg, data):
    """Ghost-padded pvar with the file's interior values (ghosts are left zero; the
    library fills them from the boundary conditions)."""
    g = lambda n: 2 if n > 1 else 0
    shape = (cfg.knum + 2 * g(cfg.knum), cfg.jnum + 2 * g(cfg.jnum), cfg.inum + 2 * g(cfg.inum))
    names = pvar_names(cfg)
    p = np.zeros((len(names),) + shape)
    sl = []
    for n in (cfg.knum, cfg.jnum, cfg.inum):
        sl.append(slice(2, -2) if n > 1 else slice(None))
    for v, name in enumerate(names):
        p[(v,) + tuple(sl)] = np.asarray(data["/timedisc/" + name]).reshape(
            cfg.knum, cfg.jnum, cfg.inum)
    return p


def save(sim, path):
    """Write a Simulation's current primitive state, time and bary centres."""
    cfg = sim.cfg
    st = sim.status()
    names = {abi.MESH_X: 0, abi.MESH_Y: 1, abi.MESH_Z: 2}
    sl = []
    for n in (cfg.knum, cfg.jnum, cfg.inum):
        sl.append(slice(2, -2) if n > 1 else slice(None))
    bary = np.stack([sim.mesh(w)[tuple(sl)] for w in names], axis=0)
    write_state(path, cfg, st.time, sim.get(abi.PVAR), bary=bary)
