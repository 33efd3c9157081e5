"""Mesh reader/writer and connectivity (Preprocess.f90 conventions)."""
import numpy as np

from lag2d_b200 import quad_mesh, read_domn, write_domn, read_ctrl, write_ctrl, Ctrl
from lag2d_b200.mesh import build_esqua, build_esuv


def test_domn_roundtrip(tmp_path):
    m = quad_mesh(5, 3, jitter=0.1, curve=0.05, seed=1)
    p = tmp_path / "dgflo2d.domn"
    write_domn(m, str(p))
    m2 = read_domn(str(p))
    assert np.array_equal(m.ipqua, m2.ipqua) and np.array_equal(m.bface, m2.bface)
    assert np.array_equal(m.coord, m2.coord)
    assert np.array_equal(m.esuv1, m2.esuv1) and np.array_equal(m.esqua, m2.esqua)


def test_ctrl_roundtrip():
    c = Ctrl(cfl=0.1, gamlg=5.0 / 3.0, ncase=1, nstag=3, tend=0.5)
    c2 = read_ctrl(write_ctrl(c))
    assert c2 == c


def test_connectivity():
    m = quad_mesh(4, 3)
    # every quad appears in the point lists of its 9 nodes, lists sorted by cell
    for e in range(m.nquad):
        for p in m.ipqua[e]:
            lst = m.esuv1[m.esuv2[p - 1]:m.esuv2[p]]
            assert e + 1 in lst and np.all(np.diff(lst) > 0)
    # face neighbours are mutual; boundary faces carry ghost ids ncell + iface
    for e in range(m.nquad):
        for k in range(4):
            j = m.esqua[e, k]
            if j <= m.ncell:
                assert e + 1 in m.esqua[j - 1]
            else:
                f = m.bface[j - m.ncell - 1]
                a, b = m.ipqua[e, k], m.ipqua[e, (k + 1) % 4]
                assert {a, b} == {f[0], f[1]}
    # the centre node satisfies the step's re-interpolation rule
    c = m.ipqua - 1
    x = m.coord[:, 0]
    assert np.allclose(x[c[:, 8]], -0.25 * x[c[:, :4]].sum(1) + 0.5 * x[c[:, 4:8]].sum(1), atol=1e-15)
    e1, e2 = build_esuv(m.iptri, m.ipqua, m.npoin)
    assert np.array_equal(e1, m.esuv1) and np.array_equal(build_esqua(m.ipqua, m.iptri, m.bface), m.esqua)
