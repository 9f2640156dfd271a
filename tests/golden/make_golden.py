"""Regenerate the oracle fixtures of tests/golden/ (run from the repository root).

Each fixture stores the ghost-padded cvar and dt of one parity case after a
few steps of the oracle.  The oracle is deterministic and compiled without FMA
contraction, so a fixture changes only if the restated algorithm changes.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from fosite_b200 import abi  # noqa: E402
from cases import CASES  # noqa: E402
import pyoracle  # noqa: E402

STEPS = 3


def main(names=None):
    """Regenerate the fixtures of the named cases (all cases without names)."""
    out = os.path.dirname(os.path.abspath(__file__))
    for name, build in sorted(CASES.items()):
        if names and name not in names:
            continue
        cfg, p, extra = build()
        o = pyoracle.Oracle(cfg)
        if "bccsound" in extra:
            o.set_sound_speeds(np.broadcast_to(extra["bccsound"], o.shape),
                               np.broadcast_to(extra["fcsound"], (4,) + o.shape))
        if "fargo_w" in extra:
            o.set_fargo_velocity(extra["fargo_w"])
        o.set_state(abi.PVAR, p)
        o.first_step()
        for _ in range(STEPS):
            o.step()
        np.savez_compressed(os.path.join(out, name + ".npz"), cvar=o.get(abi.CVAR), dt=o.status().dt, steps=STEPS)
        print(name, o.status().dt)


if __name__ == "__main__":
    main(sys.argv[1:])
