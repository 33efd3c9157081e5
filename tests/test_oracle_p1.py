"""CPU checks of the restated linear P1 branch (straight 4-node quads,
ncurv=0 / nfint=1 / nlimi=6; the reference's Sod configuration).

The reference ships no tests or outputs for this branch either.  The
restatement is pinned here by the exact solution of the Riemann problem it
is run on (a one-cell-high strip, where the radial initial rule of the Sod
case is a planar discontinuity at x = 0.5) and by the scheme's invariants:
constant cell masses, total energy conserved exactly (slip walls do no work),
and the golden fixture in tests/golden/sod12_p1.npz (tests/test_oracle.py).
"""
import numpy as np
import pytest

from lag2d_b200.config import _sod, workload
from oracle.oracle import Oracle


def _run(m, c, nsteps):
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    n, dt, ta = o.run(unkno, coord, m.coord.copy(), geoel, amatr, ustar, 1, nsteps, c.dtfix, 0.0)
    return o, geoel, amatr, unkno, coord, ustar, n, ta


def test_sod_strip_matches_exact_riemann_solution():
    """Sod (rho, p) = (1, 1) | (0.125, 0.1), gamma 1.4, at t = 0.2 on 200 x 1
    cells: the exact solution has p* = 0.30313, u* = 0.92745, post-shock
    density 0.26557, the shock at x = 0.8504, the contact at x = 0.6855 and
    the rarefaction between x = 0.2634 and 0.4859."""
    m, c = _sod(200, 1, 0.005)
    _, geoel, _, unkno, coord, _, n, ta = _run(m, c, 2000)
    assert abs(ta - 0.2) < 1e-12 and n < 2000
    nc = m.ncell
    tau, u, e = unkno[:nc, 0, 0], unkno[:nc, 1, 0], unkno[:nc, 3, 0]
    p = 0.4 / tau * (e - 0.5 * u * u)
    xc = coord[m.ipqua - 1][:, :, 0].mean(axis=1)
    left = xc < 0.15  # the rarefaction head (x = 0.2634) is smeared over a few cells
    assert np.allclose(1.0 / tau[left], 1.0, atol=1e-3) and np.allclose(p[left], 1.0, atol=1e-3)
    right = xc > 0.92  # ahead of the shock (the P1 profile decays within a few cells)
    assert np.allclose(1.0 / tau[right], 0.125, atol=1e-6) and np.allclose(u[right], 0.0, atol=1e-5)
    star = (xc > 0.58) & (xc < 0.82)  # both sides of the contact (x = 0.6855)
    assert np.abs(u[star] - 0.92745).max() < 0.03
    assert np.abs(p[star] - 0.30313).max() < 0.02
    shocked = (xc > 0.72) & (xc < 0.82)
    assert np.abs(1.0 / tau[shocked] - 0.26557).max() < 0.005
    # shock position: where the density crosses halfway between the states
    rho = 1.0 / tau
    i = np.nonzero((xc > 0.75) & (rho < 0.5 * (0.26557 + 0.125)))[0][0]
    assert abs(xc[i] - 0.8504) < 2 * 0.005
    # the plateau lies between the rarefaction tail and the shock
    assert u[(xc > 0.3) & (xc < 0.45)].max() < 0.92745


@pytest.mark.parametrize("name,nsteps", [("sod_jitter40", 40), ("sod200", 30)])
def test_p1_mass_and_energy_conservation(name, nsteps):
    m, c = workload(name)
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    nc = m.ncell
    mass = geoel[:nc, 3].copy()
    e0 = float((mass * unkno[:nc, 3, 0]).sum())
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    o.run(unkno, coord, m.coord.copy(), geoel, amatr, ustar, 1, nsteps, c.dtfix, 0.0)
    # the cell mass is the time-invariant geoel(4); the energy of the cell
    # averages moves only by rounding
    assert abs(float((mass * unkno[:nc, 3, 0]).sum()) - e0) < 1e-13 * e0
    # momentum: slip walls take the normal momentum, the interior forces cancel
    assert np.isfinite(unkno[:nc]).all()
    assert (geoel[:nc, 2] > 0).all()


def test_p1_limiter_bounds_and_slope_application():
    """On the first stage of the Sod problem the limiter coefficients lie in
    [0, 1], and the limited slopes returned in place are the unlimited ones
    scaled by aflim(1), aflim(5) and rotated by the symmetric afvec."""
    m, c = workload("sod_jitter40")
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    o.run(unkno, coord, m.coord.copy(), geoel, amatr, ustar, 1, 5, c.dtfix, 0.0)
    u0 = unkno.copy()
    rhsel, aflim, afvec = o.rhs_p1(ustar, unkno, geoel, coord)
    assert (aflim[:, [0, 3, 4]] >= 0).all() and (aflim[:, [0, 3, 4]] <= 1).all()
    assert np.array_equal(afvec[:, 1], afvec[:, 2])
    nc = m.ncell
    assert np.array_equal(unkno[:nc, :, 0], u0[:nc, :, 0])
    assert np.allclose(unkno[:nc, 0, 1:], u0[:nc, 0, 1:] * aflim[:, :1], rtol=0, atol=0)
    assert np.allclose(unkno[:nc, 3, 1:], u0[:nc, 3, 1:] * aflim[:, 4:5], rtol=0, atol=0)
    du = afvec[:, 0:1] * u0[:nc, 1, 1:] + afvec[:, 1:2] * u0[:nc, 2, 1:]
    assert np.array_equal(unkno[:nc, 1, 1:], du)
    assert np.isfinite(rhsel).all()
