"""fosite binary format (io/fileio_binary.f90): byte layout, round trip, restart state."""
import struct

import numpy as np

from fosite_b200 import abi, fileio
from cases import _khi, _gauss3d


def test_header_and_record_layout(tmp_path):
    cfg, p, _ = _khi(n=(12, 10))
    path = tmp_path / "a.bin"
    fileio.write_state(str(path), cfg, 0.25, p)
    raw = path.read_bytes()
    assert raw[:13] == b"FOSITEII\x00 8 4"
    # first record: /config/mesh/geometry, an integer
    klen = struct.unpack("<i", raw[13:17])[0]
    key = raw[17:17 + klen]
    assert key == b"/config/mesh/geometry"
    typ, nbytes, val = struct.unpack("<iii", raw[17 + klen:29 + klen])
    assert (typ, nbytes, val) == (fileio.DICT_INT, 4, abi.CARTESIAN)
    # an array record: 3 dims, byte count = data + 3 ints
    i = raw.index(b"/timedisc/density")
    typ, nbytes, d1, d2, d3 = struct.unpack("<5i", raw[i + 17:i + 37])
    assert typ == fileio.DICT_REAL_THREED and (d1, d2, d3) == (12, 10, 1) and nbytes == 12 * 10 * 8 + 12


def test_round_trip_and_restart_state(tmp_path):
    for cfg, p in (_khi(n=(12, 10))[:2], _gauss3d(n=(6, 5, 4))[:2]):
        rng = np.random.default_rng(1)
        p = p + rng.uniform(0, 1e-3, p.shape)
        path = tmp_path / "s.bin"
        bary = rng.uniform(size=(3, cfg.knum, cfg.jnum, cfg.inum))
        fileio.write_state(str(path), cfg, 1.5, p, bary=bary)
        data = fileio.read(str(path))
        assert data["/timedisc/time"] == 1.5 and data["/config/mesh/inum"] == cfg.inum
        assert np.array_equal(data["/mesh/bary_curv"], bary)
        names = fileio.pvar_names(cfg)
        assert all("/timedisc/" + n in data for n in names)
        q = fileio.restart_state(cfg, data)
        sl = [slice(None)] + [slice(2, -2) if n > 1 else slice(None) for n in (cfg.knum, cfg.jnum, cfg.inum)]
        assert np.array_equal(q[tuple(sl)], p[tuple(sl)])
        c2 = fileio.restart_config(cfg, data)
        assert c2.starttime == 1.5 and c2.inum == cfg.inum
