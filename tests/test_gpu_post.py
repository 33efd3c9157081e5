"""End-of-run output through the C-ABI (lag2d_cell_output) and the restart
pair, on the device:
  * the per-cell values (centre radius, rho, p, e_int, centre, |u|, u, v) of
    quads, triangles and the P1 path against the same formulas evaluated in
    numpy on the state lag2d_get_state returns (geterror_lag_curvhybrid
    Postprocess.f90:3700-3717, :3944-3983; geterror_lag_hybrid :3515-3582);
  * the Persson marker of the VTK file against the oracle's troubled-cell
    marks on a Sedov state;
  * a run continued from restartdg.dat + restartlag.dat against the same
    run without the interruption;
  * the VTK and profile files written from the device values."""
import dataclasses

import numpy as np
import pytest

from lag2d_b200 import post, workload
from lag2d_b200.api import Lag2DSolver
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _shp6(r, s):
    return np.array([-(1 - r - s) * (1 - 2 * (1 - r - s)), -r * (1 - 2 * r), -s * (1 - 2 * s),
                     4 * r * (1 - r - s), 4 * r * s, 4 * s * (1 - r - s)])


def _expected(m, c, unkno, coord, geoel):
    n = m.ncell
    g = c.gamlg
    xc = np.zeros(n)
    yc = np.zeros(n)
    for e in range(m.ntria):
        shp = _shp6(geoel[e, 0], geoel[e, 1])
        ids = m.iptri[e] - 1
        xc[e], yc[e] = shp @ coord[ids, 0], shp @ coord[ids, 1]
    q = m.ipqua - 1
    if m.ipqua.shape[1] == 9:
        xc[m.ntria:], yc[m.ntria:] = coord[q[:, 8], 0], coord[q[:, 8], 1]
    else:
        xc[m.ntria:] = 0.25 * coord[q[:, :4], 0].sum(axis=1)
        yc[m.ntria:] = 0.25 * coord[q[:, :4], 1].sum(axis=1)
    rho = 1.0 / unkno[:n, 0, 0]
    u, v, e = unkno[:n, 1, 0], unkno[:n, 2, 0], unkno[:n, 3, 0]
    p = (g - 1.0) * rho * (e - 0.5 * (u * u + v * v))
    return np.stack([np.hypot(xc, yc), rho, p, p / rho / (g - 1.0), xc, yc, np.hypot(u, v), u, v], axis=1)


@pytest.mark.parametrize("name,nsteps", [("tgv16", 3), ("sedov16", 4), ("tgv_hybrid16", 2), ("sod40", 5)])
def test_cell_output_matches_state(name, nsteps):
    m, c = workload(name)
    s = Lag2DSolver(m, c)
    s.init_fields()
    s.run(nsteps)
    unkno, coord, _, geoel = s.get_state()
    out, bad = s.cell_output()
    ref = _expected(m, c, unkno, coord, geoel)
    scale = np.maximum(np.abs(ref).max(axis=0), 1e-300)
    assert np.all(np.abs(out - ref) <= 1e-14 * scale), np.abs(out - ref).max(axis=0) / scale
    assert bad.shape == (m.ncell,) and set(np.unique(bad)) <= {0.0, 100.0}
    if m.ntria:
        assert np.all(bad[:m.ntria] == 0.0)
    if c.npoly == 1:
        assert np.all(bad == 0.0)
    s.close()


def test_badcell_is_the_persson_mark():
    m, c = workload("sedov16")
    c = dataclasses.replace(c, ndt=0, dtfix=2e-3)
    o = Oracle(m, c)
    g, a, u = o.init()
    x = m.coord.copy()
    us = np.zeros_like(x)
    o.run(u, x, m.coord, g, a, us, 1, 6, c.dtfix, 0.0)
    s = Lag2DSolver(m, c)
    s.init_fields()
    s.set_state(u, x, us, g, a)
    _, bad = s.cell_output()
    _, flags = Oracle(m, c).rhs(us.copy(), u.copy(), g.copy(), x, m.coord, a, 7)
    assert (flags > 0).sum() > 0
    assert np.array_equal(bad > 0, flags[:m.ncell] > 0)
    s.close()


@pytest.mark.parametrize("name", ["tgv16", "sod40", "noh_rzaw8"])
def test_restart_continues_the_run(tmp_path, name):
    """A run resumed from the restart pair equals the uninterrupted run; the
    area-weighted RZ form (nrz = 2) also restores its per-stage mass
    centre geoel(1:2), which its limiter reads first."""
    m, c = workload(name)
    a = Lag2DSolver(m, c)
    a.init_fields()
    a.run(8)
    ua, xa, _, _ = a.get_state()
    b = Lag2DSolver(m, c)
    b.init_fields()
    b.run(4)
    u, x, us, g = b.get_state()
    cen = g[:m.ncell, :2] if c.nrz == 2 else None
    post.write_restart(str(tmp_path), u[:m.ncell], x, us, b.itime, b.tacru, b.dtfix, centre=cen)
    b.close()
    u2, x2, us2, it, ta, dt, cen2 = post.read_restart(str(tmp_path), m.ncell, c.nq, c.ndegr, with_centre=True)
    assert (cen2 is None) == (cen is None)
    r = Lag2DSolver(m, c)
    g0, _, _ = r.init_fields()
    full = np.zeros((m.nsize, c.nq, c.ndegr))
    full[:m.ncell] = u2
    if cen2 is not None:
        g0[:m.ncell, :2] = cen2
        r.set_state(full, x2, us2, geoel=g0)
    else:
        r.set_state(full, x2, us2)
    r.itime, r.tacru, r.dtfix = it, ta, dt
    r.run(4)
    ur, xr, _, _ = r.get_state()
    n = m.ncell
    # restartdg.dat keeps 16 significant digits; the coordinates are exact
    # (the fields here are O(1); v vanishes on the Sod strip)
    scale = np.maximum(np.abs(ua[:n, :, 0]).max(axis=0), 1.0)
    assert np.all(np.abs(ur[:n, :, 0] - ua[:n, :, 0]).max(axis=0) <= 1e-12 * scale)
    assert np.abs(xr - xa).max() <= 1e-13
    assert abs(r.tacru - a.tacru) <= 1e-15 * a.tacru
    a.close()
    r.close()


def test_vtk_and_profile_from_device(tmp_path):
    m, c = workload("sedov16")
    s = Lag2DSolver(m, c)
    s.init_fields()
    s.run(10)
    out, bad = s.cell_output()
    _, coord, _, _ = s.get_state()
    post.write_vtk(str(tmp_path / "output.vtk"), m, coord, out, bad, ncurv=1)
    d = post.read_vtk_cell_data(str(tmp_path / "output.vtk"))
    assert np.array_equal(d["density"], out[:, 1])
    assert np.allclose(d["pressure"], out[:, 2], rtol=1e-7, atol=1e-300)
    assert np.array_equal(d["Badcell"], bad)
    path = post.write_profile(str(tmp_path), m, out, c.ncase, curved=True)
    rows = [l.split() for l in open(path).read().splitlines()]
    assert len(rows) == m.ncell
    prof = np.array([[float(t) for t in r[1:]] for r in rows])
    assert np.allclose(prof, out, rtol=1e-15, atol=1e-300)
    r, rho = post.shock_radius(out)
    # the blast has left the four centre cells and compressed a ring around them
    assert rho > 1.5 and r > 0.0
    s.close()
