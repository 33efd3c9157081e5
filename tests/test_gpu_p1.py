"""Parity of the CUDA linear P1 path (straight 4-node quads, the Sod
configuration; lag2d_p1.cu behind the same C-ABI) against the CPU oracle.

With order_exact the P1 kernels keep the reference's summation order, so the
no-FMA build (liblag2d_exact.so) must match the restatement bit for bit:
initial fields, one getrhsdg_lag_mcnew call (RHS, limited state, nodal
velocity) and whole steps.  The optimised kernels (corner faces summed per
corner, closed-form volumes, one-division limiter function) in the FMA build
stay within 1e-12 of the field scale per step.  The
limiter branches on comparisons (barthfct, the strain-rate frame), so the FMA
build is compared over a few steps only.
"""
import numpy as np
import pytest

from lag2d_b200 import workload
from lag2d_b200.api import Lag2DError, Lag2DSolver
from lag2d_b200.config import StepConfig
from lag2d_b200.mesh import linear_quad_mesh
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _field_err(a, b):
    """Max error per field relative to the field's scale; u and v share the
    velocity scale (v is rounding noise on a strip where the flow is planar)."""
    sc = [max(np.abs(b[:, q]).max(), 1e-300) for q in range(b.shape[1])]
    sc[1] = sc[2] = max(sc[1], sc[2])
    return np.array([np.abs(a[:, q] - b[:, q]).max() / sc[q] for q in range(b.shape[1])])


def _oracle_state(name, nsteps):
    m, c = workload(name)
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    _, dt, ta = o.run(unkno, coord, m.coord.copy(), geoel, amatr, ustar, 1, nsteps, c.dtfix, 0.0)
    return m, c, o, geoel, amatr, unkno, coord, ustar, dt, ta


@pytest.mark.parametrize("name", ["sod40", "sod_jitter40", "sod200"])
@pytest.mark.parametrize("exact", [True, False])
def test_p1_init_fields(name, exact):
    m, c = workload(name)
    geoel, amatr, unkno = Oracle(m, c).init()
    s = Lag2DSolver(m, c, exact=exact, order_exact=exact)
    g2, a2, u2 = s.init_fields()
    n = m.ncell
    if exact:
        for k in range(4):
            assert np.array_equal(g2[:n, k], geoel[:n, k]), k
        assert np.array_equal(a2, amatr)
        assert np.array_equal(u2[:n], unkno[:n])
        return
    for k, scale in ((0, 1.0), (1, 1.0), (2, geoel[:n, 2].max()), (3, geoel[:n, 3].max())):
        assert np.abs(g2[:n, k] - geoel[:n, k]).max() / scale < 1e-12, k
    assert np.abs(a2 - amatr).max() / np.abs(amatr).max() < 1e-11
    assert _field_err(u2[:n], unkno[:n]).max() < 1e-11


@pytest.mark.parametrize("name,nsteps", [("sod_jitter40", 4), ("sod200", 6)])
@pytest.mark.parametrize("exact", [True, False])
def test_p1_rhs_single(name, nsteps, exact):
    """One getrhsdg_lag_mcnew call on a state a few steps in: rhsel, the
    limited stage state and the new nodal velocity."""
    m, c, o, geoel, amatr, unkno, coord, ustar, _, _ = _oracle_state(name, nsteps)
    s = Lag2DSolver(m, c, exact=exact, order_exact=exact)
    s.set_state(unkno, coord, ustar, geoel, amatr)
    r2, f2 = s.rhs()
    u2, _, us2, _ = s.get_state()
    assert not f2.any()
    u1, us1 = unkno.copy(), ustar.copy()
    r1, _, _ = o.rhs_p1(us1, u1, geoel, coord)
    n = m.ncell
    if exact:
        assert np.array_equal(r2, r1)
        assert np.array_equal(u2[:n], u1[:n])
        assert np.array_equal(us2, us1)
        return
    assert _field_err(r2, r1).max() < 1e-9
    assert _field_err(u2[:n], u1[:n]).max() < 1e-11
    assert np.abs(us2 - us1).max() / np.abs(us1).max() < 1e-11


@pytest.mark.parametrize("name,nsteps", [("sod_jitter40", 12), ("sod200", 10), ("sod40", 12)])
@pytest.mark.parametrize("exact", [True, False])
def test_p1_steps(name, nsteps, exact):
    """Whole steps (getsolvdg_lag with getdelt_lag and SSP-RK2) from the
    initial state, step by step through lag2d_step."""
    m, c = workload(name)
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    s = Lag2DSolver(m, c, exact=exact, order_exact=exact)
    s.init_fields()
    dt, ta = c.dtfix, 0.0
    n = m.ncell
    for it in range(1, nsteps + 1):
        _, dt, ta = o.run(unkno, coord, m.coord.copy(), geoel, amatr, ustar, it, 1, dt, ta)
        dt2, ta2 = s.step()
        u2, x2, us2, g2 = s.get_state()
        if exact:
            assert dt2 == dt and ta2 == ta, it
            assert np.array_equal(u2[:n], unkno[:n]), it
            assert np.array_equal(x2, coord) and np.array_equal(us2, ustar), it
            assert np.array_equal(g2[:n, 2], geoel[:n, 2]), it
        else:
            assert abs(dt2 - dt) <= 1e-12 * dt, it
            assert _field_err(u2[:n, :, :1], unkno[:n, :, :1]).max() < 1e-12 * it, it
            assert np.abs(x2 - coord).max() < 1e-12, it
            # follow the oracle's state so that the bound stays per step
            s.set_state(unkno, coord, ustar, geoel, amatr)
            s.dtfix, s.tacru = dt, ta


@pytest.mark.parametrize("exact", [True, False])
def test_p1_graph_run_matches_steps(exact):
    m, c = workload("sod_jitter40")
    a = Lag2DSolver(m, c, exact=exact, order_exact=exact)
    a.init_fields()
    for _ in range(8):
        a.step()
    b = Lag2DSolver(m, c, exact=exact, order_exact=exact)
    b.init_fields()
    assert b.run(8) == 8
    ua, xa, usa, _ = a.get_state()
    ub, xb, usb, _ = b.get_state()
    assert np.array_equal(ua, ub) and np.array_equal(xa, xb) and np.array_equal(usa, usb)
    assert (a.dtfix, a.tacru) == (b.dtfix, b.tacru)


def test_p1_golden_fixture():
    """The committed oracle fixture (radial Sod on jittered 12 x 4 straight
    quads, 6 steps) reproduced bit for bit by the no-FMA build."""
    import os
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "sod12_p1.npz"))
    m = linear_quad_mesh(12, 4, 0.0, 1.0, 0.0, 0.4, jitter=0.15, seed=7)
    c = StepConfig(npoly=1, ndegr=3, mdegr=3, ncase=6, gamlg=1.4, nstag=2, cfl=0.3, tend=0.2)
    s = Lag2DSolver(m, c, exact=True, order_exact=True)
    _, a2, u0 = s.init_fields()
    n = m.ncell
    assert np.array_equal(u0[:n], ref["unkno0"][:n]) and np.array_equal(a2, ref["amatr"])
    assert s.run(int(ref["nsteps"])) == int(ref["nsteps"])
    u2, x2, us2, _ = s.get_state()
    assert np.array_equal(u2[:n], ref["unkno"][:n])
    assert np.array_equal(x2, ref["coord"]) and np.array_equal(us2, ref["ustar"])
    assert s.dtfix == float(ref["dtfix"]) and s.tacru == float(ref["tacru"])


def test_p1_energy_conservation_and_sod_run():
    """100 steps of the 200 x 10 radial Sod problem on the FMA build: cell
    masses fixed, total energy of the cell averages conserved to rounding."""
    m, c = workload("sod200")
    s = Lag2DSolver(m, c)
    g, _, u = s.init_fields()
    n = m.ncell
    mass = g[:n, 3]
    e0 = float((mass * u[:n, 3, 0]).sum())
    assert s.run(100) == 100
    u2, _, _, g2 = s.get_state()
    assert abs(float((mass * u2[:n, 3, 0]).sum()) - e0) < 1e-12 * e0
    assert np.array_equal(g2[:n, 3], mass)
    assert (g2[:n, 2] > 0).all()


def test_p1_unsupported_calls():
    m, c = workload("sod40")
    s = Lag2DSolver(m, c)
    s.init_fields()
    for call in (lambda: s.weno(np.zeros(m.ncell, np.int32)), lambda: s.adjoint(2, 1),
                 lambda: s.set_rho0(np.ones(m.ncell))):
        with pytest.raises(Lag2DError) as e:
            call()
        assert e.value.code == 3
    with pytest.raises(Lag2DError) as e:
        Lag2DSolver(m, c, precision=1)
    assert e.value.code == 3


@pytest.mark.parametrize("exact", [True, False])
def test_p1_sod_strip_to_end_time(exact):
    """The Sod strip (200 x 1 straight quads, planar discontinuity at x = 0.5)
    run to t_end = 0.2 through lag2d_run: bit for bit with the oracle in the
    reference-order no-FMA build, within 1e-10 in the optimised FMA build, and
    the star state of the exact Riemann solution (u* = 0.92745, p* = 0.30313)
    on the plateau."""
    from lag2d_b200.config import _sod
    m, c = _sod(200, 1, 0.005)
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    n1, dt1, ta1 = o.run(unkno, coord, m.coord.copy(), geoel, amatr, ustar, 1, 2000, c.dtfix, 0.0)
    s = Lag2DSolver(m, c, exact=exact, order_exact=exact)
    s.init_fields()
    assert s.run(2000) == n1 and abs(s.tacru - 0.2) < 1e-12
    u2, x2, _, _ = s.get_state()
    n = m.ncell
    if exact:
        assert np.array_equal(u2[:n], unkno[:n]) and np.array_equal(x2, coord)
    else:
        assert _field_err(u2[:n, :, :1], unkno[:n, :, :1]).max() < 1e-10
    tau, u, e = u2[:n, 0, 0], u2[:n, 1, 0], u2[:n, 3, 0]
    p = 0.4 / tau * (e - 0.5 * u * u)
    xc = x2[m.ipqua - 1][:, :, 0].mean(axis=1)
    star = (xc > 0.58) & (xc < 0.82)
    assert np.abs(u[star] - 0.92745).max() < 0.03 and np.abs(p[star] - 0.30313).max() < 0.02
