"""End-of-run output on the CPU: the Fortran edit descriptors, the restart
pair, the VTK and profile writers, and the boundary host search against a
restatement of the reference's loop (Preprocess.f90:679-717)."""
import numpy as np
import pytest

from lag2d_b200 import workload
from lag2d_b200.mesh import boundary_hosts, linear_quad_mesh, polar_mesh
from lag2d_b200 import post


def test_fortran_e_descriptor():
    assert post.fortran_e(1.0, 32, 16) == " " * 10 + "0.1000000000000000E+01"
    assert post.fortran_e(-0.0123, 20, 8) == "     -0.12300000E-01"
    assert post.fortran_e(0.0, 20, 8) == "      0.00000000E+00"
    assert len(post.fortran_e(1.23456789e-300, 32, 16)) == 32
    for x in (3.14159, -2.5e7, 1e-12):
        assert float(post.fortran_e(x, 32, 16)) == pytest.approx(x, rel=1e-15)


def _host_loop(m):
    """preprocess1 step 2 as the reference writes it: every boundary face
    against every cell's corner vertices, the last match kept."""
    hosts = np.zeros(m.nbfac, dtype=np.int32)
    for i in range(m.nbfac):
        a, b = int(m.bface[i, 0]), int(m.bface[i, 1])
        for ie in range(m.ntria):
            if sum(1 for j in (a, b) if j in m.iptri[ie, :3]) == 2:
                hosts[i] = ie + 1
        for ie in range(m.nquad):
            if sum(1 for j in (a, b) if j in m.ipqua[ie, :4]) == 2:
                hosts[i] = ie + 1 + m.ntria
    return hosts


@pytest.mark.parametrize("name", ["tgv16", "tgv_hybrid16", "noh8", "sod40"])
def test_boundary_hosts_match_reference_loop(name):
    m, _ = workload(name)
    h = boundary_hosts(m.iptri, m.ipqua, m.bface)
    assert np.array_equal(h, _host_loop(m))
    assert (h > 0).all()


def test_boundary_hosts_large_mesh_is_fast():
    import time
    m = linear_quad_mesh(512, 512)
    t = time.perf_counter()
    h = boundary_hosts(m.iptri, m.ipqua, m.bface)
    assert time.perf_counter() - t < 5.0
    # every boundary face of the structured mesh has exactly its edge cell
    assert (h > 0).all()


def test_restart_round_trip(tmp_path):
    rng = np.random.default_rng(7)
    ncell, npoin = 37, 50
    u = rng.standard_normal((ncell, 4, 6)) * 10.0 ** rng.integers(-5, 5, (ncell, 4, 6))
    x = rng.standard_normal((npoin, 2))
    us = rng.standard_normal((npoin, 2))
    post.write_restart(str(tmp_path), u, x, us, 17, 0.123, 4.5e-4)
    u2, x2, us2, it, ta, dt = post.read_restart(str(tmp_path), ncell)
    # restartdg.dat keeps 16 significant digits (E32.16), as the reference writes it
    assert np.all(np.abs(u2 - u) <= 1e-15 * np.abs(u))
    assert np.array_equal(x2, x) and np.array_equal(us2, us)
    assert (it, ta, dt) == (17, 0.123, 4.5e-4)
    lines = open(tmp_path / "restartdg.dat").read().splitlines()
    assert len(lines) == ncell * 4 * 2 and all(len(l) == 96 for l in lines)
    assert post.read_restart(str(tmp_path), ncell, with_centre=True)[6] is None
    # with the mass centres (nrz = 2): exact
    cen = rng.standard_normal((ncell, 2))
    post.write_restart(str(tmp_path), u, x, us, 17, 0.123, 4.5e-4, centre=cen)
    r = post.read_restart(str(tmp_path), ncell, with_centre=True)
    assert np.array_equal(r[6], cen) and np.array_equal(r[1], x)


def test_restart_rejects_wrong_size(tmp_path):
    post.write_restart(str(tmp_path), np.ones((3, 4, 6)), np.zeros((2, 2)), np.zeros((2, 2)), 1, 0.0, 0.0)
    with pytest.raises(ValueError):
        post.read_restart(str(tmp_path), 4)


def _fake_cellout(m, rng):
    c = rng.uniform(0.5, 2.0, (m.ncell, 9))
    c[:, 7:9] -= 1.0
    return c


def test_vtk_writer_round_trip(tmp_path):
    m, _ = workload("tgv_hybrid16")
    rng = np.random.default_rng(1)
    c = _fake_cellout(m, rng)
    bad = np.where(rng.uniform(size=m.ncell) > 0.8, 100.0, 0.0)
    path = tmp_path / "output.vtk"
    post.write_vtk(str(path), m, m.coord, c, bad, ncurv=1)
    d = post.read_vtk_cell_data(str(path))
    assert np.array_equal(d["density"], c[:, 1])
    # E20.8: 8 significant digits
    assert np.allclose(d["internalenergy"], c[:, 3], rtol=1e-7)
    assert np.allclose(d["pressure"], c[:, 2], rtol=1e-7)
    assert np.array_equal(d["Badcell"], bad)
    assert np.allclose(d["vectors"][:, :2], c[:, 7:9], rtol=1e-15)
    txt = open(path).read()
    # 7 ids per triangle row (6 nodes), 10 per quad row (9 nodes), 0-based
    assert f" CELLS {m.ncell} {7 * m.ntria + 10 * m.nquad}" in txt
    assert " CELL_TYPES" in txt and "\n 22\n" in txt and "\n 23\n" in txt


def test_profile_records():
    m = polar_mesh(4, 4)
    rng = np.random.default_rng(2)
    c = _fake_cellout(m, rng)
    recs = post.profile_lines(m, c, ncase=3)
    # Noh: triangles (7 values) then quads (9 values)
    assert len(recs) == m.ncell
    assert all(len(r) == 8 + 7 * 32 for r in recs[:m.ntria])
    assert all(len(r) == 8 + 9 * 32 for r in recs[m.ntria:])
    assert int(recs[m.ntria][:8]) == m.ntria + 1
    vals = [float(t) for t in recs[-1][8:].split()]
    assert np.allclose(vals, c[-1], rtol=1e-15)
    assert post.profile_lines(m, c, ncase=1) == []
    assert len(post.profile_lines(m, c, ncase=6)[0]) == 8 + 4 * 32
    r, rho = post.shock_radius(c)
    assert rho == c[:, 1].max()
