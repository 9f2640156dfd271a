"""Oracle pins of the benchmark configurations at their full sizes (run from the repository root).

The full states are too large to commit, so each pin keeps what a test can check a GPU run
against without re-running the oracle:
  * the SHA-256 of the interior cvar block (float64, [variable][k][j][i], little endian) --
    the --fmad=false GPU build must reproduce it bit for bit wherever no CUDA libm call
    (exp/log of absorbing boundaries) is involved;
  * per-variable sums and absolute sums over the interior (conservation, scale of the L1);
  * for the disk, whose absorbing boundaries call exp/log, every cell of the rows
    j = 7, 8 (mod 32) (all radii; rows next to the y seams of the stage tiles), against which
    the GPU state is compared in relative L1;
  * time, dt, iter and n_adj after the pinned steps.

Configurations (the benchmark's synthetic set-ups, fosite_b200.problems):
  khi256   2D KHI 256^2, SSPRK3: after FirstStep + 1 step and + 1000 steps
  disk512  logcylindrical isothermal disk 512x1024 with FARGO, absorbing r: + 1 and + 2000 steps
  gauss256 3D Gaussian pulse 256^3, Dormand-Prince: after FirstStep + 1 step (about 40 GB of
           host memory for the oracle)

  python tests/golden/make_config_pins.py [khi256] [disk512] [gauss256]
"""
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from fosite_b200 import abi, problems  # noqa: E402
import pyoracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def interior(a, cfg):
    sl = [slice(None)]
    for n in (cfg.knum, cfg.jnum, cfg.inum):
        sl.append(slice(2, -2) if n > 1 else slice(None))
    return np.ascontiguousarray(a[tuple(sl)])


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def disk_rows(cfg):
    j = np.arange(cfg.jnum)
    return j[(j % 32 == 7) | (j % 32 == 8)]


def pin(o, cfg, tag, rows=None):
    c = interior(o.get(abi.CVAR), cfg)
    st = o.status()
    flat = c.reshape(c.shape[0], -1)
    d = {tag + "_sha256": digest(c), tag + "_sum": flat.sum(axis=1), tag + "_abssum": np.abs(flat).sum(axis=1),
         tag + "_time": st.time, tag + "_dt": st.dt, tag + "_iter": st.iter, tag + "_nadj": st.n_adj}
    if rows is not None:
        d[tag + "_rows"] = c[:, rows, :] if c.ndim == 3 else c[:, 0, rows, :]
    return d


def make(name, cfg, p, extra, marks, rows=False):
    t0 = time.time()
    o = pyoracle.Oracle(cfg)
    if "bccsound" in extra:
        o.set_sound_speeds(np.broadcast_to(extra["bccsound"], o.shape),
                           np.broadcast_to(extra["fcsound"], (4,) + o.shape))
    o.set_state(abi.PVAR, p)
    o.first_step()
    out = {"threads": pyoracle.set_threads(0)}
    r = disk_rows(cfg) if rows else None
    if rows:
        out["rows_j"] = r
    done = 0
    for m in marks:
        while done < m:
            assert o.step() == 0
            done += 1
        out.update(pin(o, cfg, "s%d" % m, r))
        print(name, "steps", m, "time", o.status().time, "%.1f s" % (time.time() - t0), flush=True)
    np.savez_compressed(os.path.join(OUT, "pin_%s.npz" % name), **out)


def main(which):
    if not which or "khi256" in which:
        cfg, p, extra = problems.khi2d(n=256)
        make("khi256", cfg, p, extra, [1, 1000])
    if not which or "disk512" in which:
        cfg, p, extra = problems.disk2d(nr=512, nphi=1024, fargo=1)
        make("disk512", cfg, p, extra, [1, 2000], rows=True)
    if not which or "gauss256" in which:
        cfg, p, extra = problems.gauss3d(n=256)
        make("gauss256", cfg, p, extra, [1])


if __name__ == "__main__":
    main(sys.argv[1:])
