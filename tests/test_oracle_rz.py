"""The CPU restatement of the RZ branches of the linear P1 path (nrz = 1,
true volume; nrz = 2, area-weighted), pinned against the exact solution of
the problem they run: Noh's implosion in RZ (y the radius) is the spherical
implosion, with the shock at r = t/3, density ((gamma + 1)/(gamma - 1))^3 =
64 behind it and (1 + t/r)^2 ahead of it (gamma 5/3).  In plane geometry the
same run compresses to 16 behind the shock and (1 + t/r) ahead of it, so
the radius weights are checked too."""
import dataclasses

import numpy as np
import pytest

from lag2d_b200 import workload
from oracle.oracle import Oracle


def _run_to_end(name, nrz=None):
    import dataclasses
    m, c = workload(name)
    if nrz is not None:
        c = dataclasses.replace(c, nrz=nrz)
    o = Oracle(m, c)
    g, a, u = o.init()
    x = m.coord.copy()
    us = np.zeros_like(x)
    it, dt, tac = 1, c.dtfix, 0.0
    Oracle.status()  # reads and clears what earlier calls left
    while tac < c.tend * (1.0 - 1e-12):
        done, dt, tac = o.run(u, x, m.coord, g, a, us, it, 50, dt, tac)
        assert Oracle.status() == 0 and np.isfinite(dt)
        it += done
        if done < 50:
            break
    n = m.ncell
    ctr = np.array([x[m.ipqua[i] - 1].mean(axis=0) for i in range(n)])
    return m, c, tac, 1.0 / u[:n, 0, 0], np.hypot(ctr[:, 0], ctr[:, 1]), ctr


def test_rz_initial_volumes_carry_the_radius():
    m, c = workload("noh_rz8")
    g, a, u = Oracle(m, c).init()
    n = m.ncell
    ctr = np.array([m.coord[m.ipqua[i] - 1].mean(axis=0) for i in range(n)])
    h = 1.0 / 8
    # true volume per radian of a straight square cell: h^2 times its centre radius
    assert np.allclose(g[:n, 2], h * h * ctr[:, 1], rtol=1e-13)
    assert abs(g[:n, 2].sum() - 0.5) < 1e-14
    # rho = 1: mass equals volume, and the mass centre sits above the centroid
    assert np.allclose(g[:n, 3], g[:n, 2], rtol=1e-13)
    assert np.all(g[:n, 1] >= -1e-15)


@pytest.mark.parametrize("name", ["noh_rz32", "noh_rzaw32"])
def test_rz_noh_spherical_solution(name):
    m, c, t, rho, r, ctr = _run_to_end(name)
    assert abs(t - 0.6) < 1e-12
    shocked = (r > 0.1) & (r < 0.15)
    assert 50.0 < rho[shocked].mean() < 68.0  # exact 64 (32 x 32: 55.4 true volume, 52.4 area-weighted)
    # ahead of the shock, away from the free outer sides' rarefaction
    ahead = (r > 0.4) & (r < 0.7) & (ctr.max(axis=1) < 0.75)
    exact = (1.0 + t / r[ahead]) ** 2
    assert np.abs(rho[ahead] / exact - 1.0).mean() < 0.05
    # the shock has passed r = 0.15 and not reached r = 0.3
    assert rho[(r > 0.3) & (r < 0.4)].max() < 20.0


def test_plane_noh_on_the_same_mesh_is_cylindrical():
    m, c, t, rho, r, ctr = _run_to_end("noh_rz32", nrz=0)
    ahead = (r > 0.4) & (r < 0.7) & (ctr.max(axis=1) < 0.75)
    exact = 1.0 + t / r[ahead]
    assert np.abs(rho[ahead] / exact - 1.0).mean() < 0.05
    assert 12.0 < rho[(r > 0.1) & (r < 0.15)].mean() < 18.0  # exact 16


def test_rzaw_initial_geometry_is_area_based():
    """nrz = 2 (GetInitial.f90:1655-1691, :604-675): the mass and the mass
    centre are taken over the area, geoel(3) stays the true volume, geoel(11)
    is volume / area (the centroid radius of a straight square cell), and
    M^-1 is the area mass matrix's inverse divided by geoel(11)."""
    m, c = workload("noh_rzaw8")
    g, a, u = Oracle(m, c).init()
    g1, a1, _ = Oracle(m, dataclasses.replace(c, nrz=0)).init()
    n = m.ncell
    ctr = np.array([m.coord[m.ipqua[i] - 1].mean(axis=0) for i in range(n)])
    h = 1.0 / 8
    assert np.allclose(g[:n, 2], h * h * ctr[:, 1], rtol=1e-13)
    assert np.allclose(g[:n, 3], h * h, rtol=1e-13)
    assert np.allclose(g[:n, 10], ctr[:, 1], rtol=1e-13)
    # rho = 1: the area mass centre is the centroid, as in plane geometry
    assert np.allclose(g[:n, :2], g1[:n, :2], atol=1e-14)
    assert np.allclose(a * g[:n, 10:11], a1, rtol=1e-13)
