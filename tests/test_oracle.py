"""CPU checks of the oracle (the checker the GPU path is measured against).

The reference cannot run here (Fortran, no compiler), so the oracle is pinned
by properties the reference scheme has by construction and by its own golden
fixtures: exact per-cell mass, total energy, free-stream preservation,
quadratic reproduction of the WENO reconstruction, symmetry, and the
committed fixtures of tests/golden/.
"""
import os

import numpy as np
import pytest

from lag2d_b200.config import noh_parity_config
from lag2d_b200.mesh import hybrid_mesh, polar_mesh
from lag2d_b200 import quad_mesh, StepConfig, workload
from oracle.oracle import Oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _run(m, c, nsteps):
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    n, dt, ta = o.run(unkno, coord, m.coord, geoel, amatr, ustar, 1, nsteps, c.dtfix, 0.0)
    return o, geoel, amatr, unkno, coord, ustar, dt, ta


def test_init_geometry_uniform():
    m = quad_mesh(4, 4, 0.0, 2.0, 0.0, 1.0)
    c = StepConfig(ncase=7, sedov_cells=())
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    n = m.ncell
    assert np.allclose(geoel[:n, 2], 0.5 * 0.25, rtol=1e-14)   # volume
    assert np.allclose(geoel[:n, 3], geoel[:n, 2], rtol=1e-14)  # mass (rho0 = 1)
    assert np.abs(geoel[:n, :2]).max() < 1e-15                 # mass centre at the reference origin
    # P2 offsets: 0.5 * <r^2> = 1/6 on the reference square
    assert np.allclose(geoel[:n, 18], 1.0 / 6.0, rtol=1e-14)
    assert np.allclose(geoel[:n, 19], 1.0 / 6.0, rtol=1e-14)
    assert np.abs(geoel[:n, 20]).max() < 1e-15
    # tau average = V / m = 1
    assert np.allclose(unkno[:n, 0, 0], 1.0, rtol=1e-14)


def test_mass_matrix_inverse():
    m = quad_mesh(3, 3, jitter=0.1, curve=0.05, seed=2)
    c = StepConfig(ncase=7, sedov_cells=())
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    assert np.allclose(amatr[:, 15], 1.0 / geoel[:m.ncell, 3], rtol=1e-13)
    # the 5x5 block is symmetric positive definite
    for e in range(m.ncell):
        M = np.zeros((5, 5))
        k = 0
        for i in range(5):
            for j in range(i, 5):
                M[i, j] = M[j, i] = amatr[e, k]
                k += 1
        assert np.linalg.eigvalsh(M).min() > 0


# on the tri/quad mesh the Taylor-Green source integrates to zero over the box
# only up to the error of the 7-point triangle rule (~1e-13 of the energy)
@pytest.mark.parametrize("name,nsteps,tol", [("tgv16", 15, 1e-13), ("sedov16", 15, 1e-13), ("tgv_hybrid16", 10, 1e-12),
                                           ("noh8", 10, 1e-13)])
def test_mass_and_energy_conservation(name, nsteps, tol):
    m, c = workload(name)
    if name.startswith("noh"):
        c = noh_parity_config(c)
    o, geoel, amatr, unkno, coord, ustar, dt, ta = _run(m, c, nsteps)
    n = m.ncell
    o.cellvol(geoel, coord)
    # The cell mass m is fixed (amatr(16) = 1/m never changes).  The discrete
    # geometric conservation law V(x) = m * tau_bar holds up to the scheme's
    # truncation error only (Simpson-weighted sub-cell face fluxes versus a
    # 6x6 Gauss volume of the curved cell), so it is a sanity bound here.
    gcl = np.abs(geoel[:n, 2] - geoel[:n, 3] * unkno[:n, 0, 0]).max() / geoel[:n, 2].max()
    assert gcl < 1e-3, gcl
    geoel0, _, u0 = Oracle(m, c).init()
    e0 = (geoel0[:n, 3] * u0[:n, 3, 0]).sum()
    e1 = (geoel[:n, 3] * unkno[:n, 3, 0]).sum()
    assert abs(e1 - e0) / abs(e0) < tol
    assert not np.isnan(unkno).any()


def test_free_stream_preservation():
    m = quad_mesh(6, 6, jitter=0.15, curve=0.1, seed=3)
    c = StepConfig(ncase=7, gamlg=1.4, sedov_cells=())
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    bnodes = set((m.bface[:, [0, 1, 4]].reshape(-1) - 1).tolist())
    inner_nodes = np.array([i for i in range(m.npoin) if i not in bnodes])
    cells = [e for e in range(m.ncell) if not any((n - 1) in bnodes for n in m.ipqua[e])]
    for U, V in [(0.0, 0.0), (0.3, -0.7)]:
        u = np.zeros_like(unkno)
        u[:, 0, 0] = 1.0
        u[:, 1, 0], u[:, 2, 0] = U, V
        u[:, 3, 0] = 1.0 / 0.4 + 0.5 * (U * U + V * V)
        ustar = np.zeros_like(m.coord)
        ustar[:, 0], ustar[:, 1] = U, V
        r, flags = o.rhs(ustar, u, geoel.copy(), m.coord.copy(), m.coord, amatr)
        assert np.abs(ustar[inner_nodes] - [U, V]).max() < 1e-14
        assert np.abs(r[cells]).max() < 1e-14
        assert flags.sum() == 0


def test_weno_reproduces_quadratics_on_uniform_mesh():
    m = quad_mesh(8, 8)
    c = StepConfig(ncase=7, gamlg=1.4, sedov_cells=())
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coef = [(1.0, 0.1, -0.05, 0.02, 0.03, -0.01), (0.5, 0.2, 0.1, -0.1, 0.05, 0.02),
            (0.3, -0.1, 0.2, 0.05, -0.02, 0.04), (3.0, 0.3, 0.2, 0.1, -0.1, 0.05)]
    h = 1.0 / 8
    u = np.zeros_like(unkno)
    for e in range(m.ncell):
        xc, yc = m.coord[m.ipqua[e, 8] - 1]
        for q, cf in enumerate(coef):
            # exact Taylor moments of a quadratic on an affine square (r = (x-xc)/(h/2))
            a, b, cc, d, ee, f = cf
            s = h / 2
            val = a + b * xc + cc * yc + d * xc * xc + ee * xc * yc + f * yc * yc
            gx, gy = b + 2 * d * xc + ee * yc, cc + ee * xc + 2 * f * yc
            hxx, hyy, hxy = 2 * d * s * s, 2 * f * s * s, ee * s * s
            u[e, q, 0] = val + 0.5 * hxx * (1.0 / 3.0) + 0.5 * hyy * (1.0 / 3.0)
            u[e, q, 1], u[e, q, 2] = gx * s, gy * s
            u[e, q, 3], u[e, q, 4], u[e, q, 5] = hxx, hyy, hxy
    flags = np.zeros(m.ncell, dtype=np.int32)
    interior = [e for e in range(m.ncell) if 0 < e % 8 < 7 and 0 < e // 8 < 7]
    flags[interior] = 1
    u2 = u.copy()
    o.weno(u2, geoel.copy(), m.coord.copy(), m.coord, flags)
    assert Oracle.status() == 0
    assert np.abs(u2 - u).max() < 1e-13
    # a troubled domain-corner cell hits the reference's stencil `stop`
    flags[:] = 0
    flags[0] = 1
    o.weno(u.copy(), geoel.copy(), m.coord.copy(), m.coord, flags)
    assert Oracle.status() == 2


def test_tgv_symmetry():
    m, c = workload("tgv16")
    o, geoel, amatr, unkno, coord, ustar, dt, ta = _run(m, c, 5)
    n = 16
    tau = unkno[:m.ncell, 0, 0].reshape(n, n)
    # The Taylor-Green vortex is invariant under the quarter turn about the
    # domain centre, which maps each quad's corner k to corner k+1: the scheme's
    # sub-cell tables are cyclic, so the discrete field keeps the symmetry.
    # (It is not mirror-symmetric: the two faces of a corner carry different
    # weights, Getrhslaggauss.f90:10534-10552.)
    assert np.abs(tau - np.rot90(tau, -1)).max() < 1e-12


@pytest.mark.parametrize("name", ["tgv8", "sedov12", "tgv6_curved", "tgv6_hybrid", "noh4_polar", "sod12_p1"])
def test_golden_fixtures(name):
    from tests.golden.make_golden import run_case
    ref = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    got = run_case(name)
    for k in ("unkno0", "amatr", "unkno", "coord", "ustar"):
        scale = max(np.abs(ref[k]).max(), 1e-300)
        assert np.abs(got[k] - ref[k]).max() / scale < 1e-14, k
    assert abs(float(got["dtfix"]) - float(ref["dtfix"])) <= 1e-15 * float(ref["dtfix"])


def test_free_stream_preservation_hybrid():
    """Uniform states stay uniform on a jittered, curved tri/quad mesh: the
    triangle sub-cell normals and weights close like the quad ones."""
    m = hybrid_mesh(6, 6, jitter=0.15, curve=0.1, seed=3)
    c = StepConfig(ncase=7, gamlg=1.4, sedov_cells=())
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    bnodes = set((m.bface[:, [0, 1, 4]].reshape(-1) - 1).tolist())
    inner = np.array([i for i in range(m.npoin) if i not in bnodes])
    conn = [m.iptri[i] for i in range(m.ntria)] + [m.ipqua[i] for i in range(m.nquad)]
    cells = [e for e in range(m.ncell) if not any((n - 1) in bnodes for n in conn[e])]
    assert any(e < m.ntria for e in cells) and any(e >= m.ntria for e in cells)
    for U, V in [(0.0, 0.0), (0.3, -0.7)]:
        u = np.zeros_like(unkno)
        u[:, 0, 0] = 1.0
        u[:, 1, 0], u[:, 2, 0] = U, V
        u[:, 3, 0] = 1.0 / 0.4 + 0.5 * (U * U + V * V)
        ustar = np.zeros_like(m.coord)
        ustar[:, 0], ustar[:, 1] = U, V
        r, flags = o.rhs(ustar, u, geoel.copy(), m.coord.copy(), m.coord, amatr)
        assert np.abs(ustar[inner] - [U, V]).max() < 1e-14
        assert np.abs(r[cells]).max() < 1e-14
        assert flags.sum() == 0


def test_hybrid_mesh_geometry():
    """Triangle cells of the hybrid mesh: exact areas (straight sides), total
    area of the box, mass matrix SPD."""
    m = hybrid_mesh(4, 4, 0.0, 1.0, 0.0, 1.0)
    assert m.ntria == 16 and m.nquad == 8
    c = StepConfig(ncase=1, gamlg=5.0 / 3.0)
    geoel, amatr, unkno = Oracle(m, c).init()
    n = m.ncell
    assert abs(geoel[:n, 2].sum() - 1.0) < 1e-14
    assert np.allclose(geoel[:m.ntria, 2], 1.0 / 32.0, rtol=0, atol=1e-15)
    for e in range(m.ntria):
        M = np.zeros((5, 5))
        k = 0
        for i in range(5):
            for j in range(i, 5):
                M[i, j] = M[j, i] = amatr[e, k]
                k += 1
        assert np.linalg.eigvalsh(M).min() > 0


def test_polar_mesh_geometry():
    """Quarter-disk mesh of the Noh workload: every node used, curved cells
    of positive volume whose total is the quarter disk up to the quadratic
    arc interpolation (O(h^4)), SPD mass matrices, face neighbours paired."""
    m = polar_mesh(8, 8)
    assert m.ntria == 8 and m.nquad == 56
    used = set(m.ipqua.reshape(-1).tolist()) | set(m.iptri.reshape(-1).tolist())
    assert used == set(range(1, m.npoin + 1))
    c = StepConfig(ncase=3, gamlg=5.0 / 3.0)
    geoel, amatr, unkno = Oracle(m, c).init()
    n = m.ncell
    assert (geoel[:n, 2] > 0).all()
    assert abs(geoel[:n, 2].sum() - np.pi / 4) < 1e-4
    for e in range(n):
        M = np.zeros((5, 5))
        k = 0
        for i in range(5):
            for j in range(i, 5):
                M[i, j] = M[j, i] = amatr[e, k]
                k += 1
        assert np.linalg.eigvalsh(M).min() > 0
    # quad face neighbours: interior faces point back, boundary faces carry ghost ids
    for q in range(m.nquad):
        for k in range(4):
            nb = m.esqua[q, k]
            assert nb > 0
            if m.ntria < nb <= n:
                assert m.ntria + q + 1 in m.esqua[nb - m.ntria - 1]
    # the Noh state: inward unit velocity, p = 1e-6
    u, v = unkno[:n, 1, 0], unkno[:n, 2, 0]
    assert np.abs(np.hypot(u, v) - 1.0).max() < 0.05


def test_initial_density_factors():
    """The per-cell initial-density hook scales the cell mass (uniform base
    density), keeps the volumes, and sets tau = 1/rho0 in the cell averages
    while pressure and velocity stay those of the case."""
    from lag2d_b200.config import initial_density_factors
    m, c = workload("sedov_hybrid_jitter16")
    f = initial_density_factors(m)
    g0, a0, u0 = Oracle(m, c).init()
    g1, a1, u1 = Oracle(m, c, rho0=f).init()
    n = m.ncell
    assert np.allclose(g1[:n, 2], g0[:n, 2], rtol=1e-14, atol=0)
    assert np.allclose(g1[:n, 3], f * g0[:n, 3], rtol=1e-13, atol=0)
    assert np.allclose(u1[:n, 0, 0], u0[:n, 0, 0] / f, rtol=1e-13, atol=0)
    p0 = (c.gamlg - 1.0) / u0[:n, 0, 0] * (u0[:n, 3, 0] - 0.5 * (u0[:n, 1, 0] ** 2 + u0[:n, 2, 0] ** 2))
    p1 = (c.gamlg - 1.0) / u1[:n, 0, 0] * (u1[:n, 3, 0] - 0.5 * (u1[:n, 1, 0] ** 2 + u1[:n, 2, 0] ** 2))
    assert np.allclose(p1, p0, rtol=1e-11, atol=1e-17)


def test_error_norms_third_order_projection():
    """geterror_lag_curvhybrid's L2 errors of the initial Taylor-Green P2
    projection fall by ~8x per mesh halving (third order) for |u| and p, and
    the density error is rounding (the projection of rho = 1)."""
    from lag2d_b200.config import _tgv
    errs = []
    for n in (8, 16, 32):
        m, c = _tgv(n)
        o = Oracle(m, c)
        geoel, _, unkno = o.init()
        errs.append(o.error_norms(unkno, geoel, m.coord))
    errs = np.array(errs)
    assert (errs[:, 0] < 1e-13).all()
    for k in (1, 2):
        ratios = errs[:-1, k] / errs[1:, k]
        assert (ratios > 7.5).all() and (ratios < 8.5).all(), ratios
