"""Stage-kernel tile layouts against the CPU oracle.

The stage kernel comes in several tile layouts (shared-memory tiles 0/2/3/4/5, the
warp-shuffle window 1, the tile whose halo planes arrive by TMA bulk tensor copies 6),
picked per grid by the tuner; FGPU_STAGE_VARIANT / FGPU_KCHUNK force one.  Every layout
must give the oracle's numbers bit for bit on the --fmad=false build, and the product
build must stay within 1e-12 relative L1 of it.  The TMA layout applies FARGO's frame
changes where it converts the staged points; launches it does not serve (viscosity,
accretion, odd x extent) run on layout 0, and those cases check that the fallback keeps
the results too.
"""
import numpy as np
import pytest

from fosite_b200 import abi
from cases import CASES, _gauss3d
from test_gpu_parity import _compare, _inexact, _interior, _pair, rel_l1

pyoracle = pytest.importorskip("pyoracle")


def _force(monkeypatch, variant, kchunk=None):
    monkeypatch.setenv("FGPU_STAGE_VARIANT", str(variant))
    if kchunk:
        monkeypatch.setenv("FGPU_KCHUNK", str(kchunk))
    else:
        monkeypatch.delenv("FGPU_KCHUNK", raising=False)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_layout_bitwise(name, monkeypatch):
    """RHS, FirstStep's dt and four steps of the TMA layout equal the oracle's bit for bit."""
    _force(monkeypatch, 6, 4)
    cfg, o, g = _pair(name, exact=True)
    tol = 1e-13 if _inexact(cfg) else 0.0
    o.compute_rhs()
    rg = _interior(g.compute_rhs(), cfg)
    ro = _interior(o.get(abi.RHS), cfg)
    if tol == 0.0:
        bad = np.argwhere(rg != ro)
        assert bad.size == 0, "rhs: %d cells differ, first %s gpu=%r oracle=%r" % (
            len(bad), bad[0], rg[tuple(bad[0])], ro[tuple(bad[0])])
    else:
        assert rel_l1(rg, ro) <= tol
    g.close()
    # a fresh pair for the steps: with FARGO the oracle's ComputeRHS frames cvar in place (its
    # rounding stays in the state), fgpu_compute_rhs leaves the stored state untouched
    cfg, o, g = _pair(name, exact=True)
    assert o.first_step() == 0
    assert g.first_step() == 0
    for s in range(4):
        ro_, rg_ = o.step(), g.step()
        assert ro_ == rg_
        so, sg = o.status(), g.status()
        assert sg.iter == so.iter and sg.n_adj == so.n_adj
        if tol == 0.0:
            assert sg.time == so.time and sg.dt == so.dt, (s, sg.time, so.time, sg.dt, so.dt)
        _compare(cfg, o, g, tol, "step %d" % s)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_2d_tile_columns_bitwise(name, monkeypatch):
    """2D blocks computing columns of three TMA tiles (the next tile's box in flight, the last
    column partial where the tile rows do not divide): four steps equal the oracle's bit for
    bit on the exact build."""
    _force(monkeypatch, 6)
    monkeypatch.setenv("FGPU_TMA_TPB", "3")
    cfg, o, g = _pair(name, exact=True)
    if cfg.knum > 1:
        g.close()
        pytest.skip("3D case: z-marching tiles")
    tol = 1e-13 if _inexact(cfg) else 0.0
    assert o.first_step() == 0
    assert g.first_step() == 0
    for s in range(4):
        assert o.step() == g.step()
        so, sg = o.status(), g.status()
        assert sg.iter == so.iter and sg.n_adj == so.n_adj
        if tol == 0.0:
            assert sg.time == so.time and sg.dt == so.dt, (s, sg.time, so.time)
        _compare(cfg, o, g, tol, "step %d" % s)
    g.close()


# 3D Dormand-Prince with at least three tiles (x: 32-wide tiles, y: 4- or 8-high tiles, z:
# chunks of 16) in every direction, reflecting walls and a Gaussian pulse
def _multi_tile():
    return _gauss3d(n=(72, 40, 40), seed=73)


_REF = {}


def _multi_tile_reference(steps):
    if steps not in _REF:
        cfg, p, _ = _multi_tile()
        o = pyoracle.Oracle(cfg)
        o.set_state(abi.PVAR, p)
        o.first_step()
        for _ in range(steps):
            assert o.step() == 0
        st = o.status()
        _REF[steps] = (o.get(abi.CVAR), o.get(abi.PVAR), st.time, st.dt, st.iter, st.n_adj)
    return _REF[steps]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
def test_multi_tile_3d_every_layout(variant, monkeypatch):
    """72x40x40 Dormand-Prince, two steps, z chunk 16: bit for bit on the exact build."""
    from fosite_b200.sim import Simulation
    _force(monkeypatch, variant, 16)
    cfg, p, _ = _multi_tile()
    c_ref, p_ref, t_ref, dt_ref, it_ref, adj_ref = _multi_tile_reference(2)
    g = Simulation(cfg, exact=True)
    assert g.stage_layout()[0] == variant
    g.set_state(abi.PVAR, p)
    g.first_step()
    for _ in range(2):
        assert g.step() == 0
    st = g.status()
    assert (st.time, st.dt, st.iter, st.n_adj) == (t_ref, dt_ref, it_ref, adj_ref)
    for got, ref, nm in ((g.get(abi.CVAR), c_ref, "cvar"), (g.get(abi.PVAR), p_ref, "pvar")):
        a, b = _interior(got, cfg), _interior(ref, cfg)
        bad = np.argwhere(a != b)
        assert bad.size == 0, "%s: %d cells differ, first %s" % (nm, len(bad), bad[0])
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [4, 6])
def test_multi_tile_3d_product_build(variant, monkeypatch):
    """The product build of the same case within 1e-12 relative L1 after one and two steps."""
    from fosite_b200.sim import Simulation
    _force(monkeypatch, variant, 16)
    cfg, p, _ = _multi_tile()
    g = Simulation(cfg, exact=False)
    g.set_state(abi.PVAR, p)
    g.first_step()
    for s in (1, 2):
        assert g.step() == 0
        ref = _multi_tile_reference(s)[0]
        r = rel_l1(_interior(g.get(abi.CVAR), cfg), _interior(ref, cfg))
        assert r <= 1e-12, (s, r)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["khi_ssprk3_mc_prim", "disk_logcyl_pointmass", "iso_axis_cyl3d"])
@pytest.mark.parametrize("variant", [0, 6])
@pytest.mark.parametrize("exact", [True, False])
def test_shu_osher_formed_primitive_states(name, variant, exact, monkeypatch):
    """Fixed-step Shu-Osher with primitive reconstruction: stages 1 and 2 also write the
    primitive variables of their results, which the next stage reads ready-made; the states
    after six steps equal those of converting every staged point (FGPU_FORM_SO=0) bit for bit,
    on the shared-memory and the TMA-staged tiles, exact and product builds."""
    from fosite_b200.sim import Simulation
    _force(monkeypatch, variant)
    out = []
    for form in ("1", "0"):
        monkeypatch.setenv("FGPU_FORM_SO", form)
        cfg, p, extra = CASES[name]()
        g = Simulation(cfg, exact=exact)
        if "bccsound" in extra:
            g.set_sound_speeds(np.broadcast_to(extra["bccsound"], g.shape),
                               np.broadcast_to(extra["fcsound"], (4,) + g.shape))
        g.set_state(abi.PVAR, p)
        g.first_step()
        assert g.run(6)[1] == 6
        out.append((g.get(abi.CVAR), g.status().time))
        g.close()
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
