"""Initial-data helpers that need the right-hand side of the scheme.

`centrifugal_velocity` restates timedisc_base%GetCentrifugalVelocity
(timedisc_base.f90:2355-2530): the velocity of a rotating flow in equilibrium
between the centrifugal force and the accelerations the scheme itself produces
(pressure gradient, gravity, geometric terms).  fosite's disk setups use it to
balance their initial rotation (e.g. examples/mmsn.f90:305).  One ComputeRHS of
the current state gives the acceleration a = -rhs_momentum / density; with
omega the rotation axis (default z), d the position vector's component
perpendicular to the axis and e_phi = omega x d/|d|:

    v = sqrt(max(0, -sum_k a_k d_k)) * e_phi

The arithmetic follows the reference's order (vector sums in component order).
The right-hand side comes from `Simulation.compute_rhs` (or the oracle's), i.e.
ComputeRHS without the CHECK_PMIN round trip; the state must be uploaded (and,
for locally isothermal disks, the sound speeds set) first.
"""
import numpy as np

from . import abi


def _curvilinear_position(cfg, mesh):
    """Mesh%posvec%bcenter and the curvilinear components of e_z, both [3, KG, JG, IG]."""
    if cfg.geometry in (abi.CYLINDRICAL, abi.LOGCYLINDRICAL):
        r = mesh(abi.MESH_RADIUS)
        z = mesh(abi.MESH_Z)
        pos = np.stack([r, np.zeros_like(r), z])
        eom = np.stack([np.zeros_like(r), np.zeros_like(r), np.ones_like(r)])
    elif cfg.geometry == abi.CARTESIAN:
        pos = np.stack([mesh(abi.MESH_X), mesh(abi.MESH_Y), mesh(abi.MESH_Z)])
        eom = np.zeros_like(pos)
        eom[2] = 1.0
    else:
        raise ValueError("geometry not supported")
    return pos, eom


def centrifugal_velocity(cfg, mesh, rhs, pvar):
    """Velocity field [VDIM, KG, JG, IG] balancing the accelerations in rhs.

    cfg: the run's config; mesh: callable returning a ghost-padded coordinate array
    (e.g. Simulation.mesh); rhs / pvar: ghost-padded arrays [V, KG, JG, IG] of the
    right-hand side and the primitive state.
    """
    pos, eom = _curvilinear_position(cfg, mesh)
    # remove the component along the axis: d = pos - (pos.e) e
    t = pos[0] * eom[0] + pos[1] * eom[1] + pos[2] * eom[2]
    d = np.stack([pos[k] - t * eom[k] for k in range(3)])
    t = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    bx, by, bz = d[0] / t, d[1] / t, d[2] / t
    ax, ay, az = eom[0], eom[1], eom[2]
    ephi = np.stack([ay * bz - az * by, az * bx - ax * bz, ax * by - ay * bx])
    comps = [k for k, n in enumerate((cfg.inum, cfg.jnum, cfg.knum)) if n > 1]
    vdim = len(comps)
    accel = [-rhs[1 + l] / pvar[0] for l in range(vdim)]
    s = accel[0] * d[comps[0]]
    for l in range(1, vdim):
        s = s + accel[l] * d[comps[l]]
    t = np.sqrt(np.maximum(0.0, -s))
    return np.stack([t * ephi[comps[l]] for l in range(vdim)])


def balance_rotation(sim, pvar):
    """Upload pvar, evaluate the RHS on the device and return pvar with its velocity
    replaced by the centrifugal-equilibrium velocity (fosite's disk set-up pattern)."""
    sim.set_state(abi.PVAR, pvar)
    rhs = sim.compute_rhs()
    v = centrifugal_velocity(sim.cfg, sim.mesh, rhs, pvar)
    out = np.array(pvar, dtype=np.float64, copy=True)
    out[1:1 + v.shape[0]] = v
    return out
