"""The WENO part of the adjoint, through the C-ABI.

With its active set frozen (Persson marks, stencils, nonlinear weights,
velocity frame and characteristic matrices taken at the state), the WENO
reconstruction is a linear map M of the DOFs (lag2d_weno_linear); the
adjoint applies M^T at every RK stage.  Checked here on a Sedov state where
WENO replaces cells:
  * M(U) at the state U is the reconstruction itself (the step's WENO pass),
    to 1e-12 of each field's scale;
  * M^T is the transpose of M: <M v, w> = <v, M^T w> to 1e-12 relative, for
    seeded random v, w;
  * lag2d_adjoint runs on windows in which WENO replaces cells (it used to
    return LAG2D_EUNSUP there), with finite gradients that agree across
    checkpoint intervals to 1e-12 of their scale, and the frozen-limiter
    directional derivatives agree with central differences of the full step
    in directions that leave the troubled cells' stencils alone.
"""
import dataclasses

import numpy as np
import pytest

from lag2d_b200 import workload
from lag2d_b200.api import Lag2DSolver
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _sedov_state(nsteps=6, drift=0.0, lift=0.0, jitter=0.0):
    """Sedov 16x16 after nsteps oracle steps at a fixed dt: Persson marks
    quads behind the shock and WENO replaces them.  drift adds a uniform x
    velocity to the initial cell averages, with the kinetic energy it
    carries, so that every cell moves (Persson then also marks the quads at
    the x walls; their stencils are incomplete and they stay unlimited).
    lift adds specific internal energy to every cell: the ambient pressure
    of the Sedov problem, 1e-6, is exactly the pressure floor max(1e-6, p)
    of the corner and volume terms, where the step is not differentiable
    (a central difference there averages the two one-sided derivatives).
    jitter adds seeded random cell-average velocities of that size, with the
    kinetic energy they carry: in a uniform drift the velocity jump |du . n|
    of the corner impedances is exactly zero on every face parallel to the
    drift, the kink of |.|, where the adjoint takes one side and a central
    difference neither."""
    m, c = workload("sedov16")
    c = dataclasses.replace(c, ndt=0, dtfix=2e-3)
    o = Oracle(m, c)
    g, a, u = o.init()
    n = m.ncell
    if drift:
        u[:n, 1, 0] += drift
        u[:n, 3, 0] += 0.5 * drift ** 2
    if lift:
        u[:n, 3, 0] += lift
    if jitter:
        rng = np.random.default_rng(3)
        du = jitter * rng.standard_normal((n, 2))
        ke0 = 0.5 * (u[:n, 1, 0] ** 2 + u[:n, 2, 0] ** 2)
        u[:n, 1, 0] += du[:, 0]
        u[:n, 2, 0] += du[:, 1]
        u[:n, 3, 0] += 0.5 * (u[:n, 1, 0] ** 2 + u[:n, 2, 0] ** 2) - ke0
    x = m.coord.copy()
    us = np.zeros_like(x)
    o.run(u, x, m.coord, g, a, us, 1, nsteps, c.dtfix, 0.0)
    return m, c, g, a, u, x, us


def _solver(m, c, g, a, u, x, us):
    s = Lag2DSolver(m, c)
    s.init_fields()
    s.set_state(u, x, us, g, a)
    return s


def test_frozen_map_is_the_reconstruction():
    m, c, g, a, u, x, us = _sedov_state()
    n = m.ncell
    s = _solver(m, c, g, a, u, x, us)
    mu = s.weno_linear(u[:n])
    ref = _solver(m, c, g, a, u, x, us)
    _, flags = ref.rhs(itime=7)
    limited = ref.get_state()[0]
    assert flags.sum() > 0
    changed = np.abs(limited[:n] - u[:n]).max(axis=(1, 2)) > 0
    assert changed.sum() > 0, "WENO replaced no cell"
    for q in range(4):
        scale = np.abs(limited[:n, q, :]).max()
        assert np.abs(mu[:n, q, :] - limited[:n, q, :]).max() <= 1e-12 * scale, q
    s.close()
    ref.close()


def test_transpose_dot_product():
    m, c, g, a, u, x, us = _sedov_state()
    n = m.ncell
    s = _solver(m, c, g, a, u, x, us)
    rng = np.random.default_rng(11)
    for _ in range(3):
        v = rng.standard_normal((n, 4, 6))
        w = rng.standard_normal((n, 4, 6))
        mv = s.weno_linear(v)[:n]
        mtw = s.weno_linear(w, transpose=True)[:n]
        lhs, rhs = float(np.sum(mv * w)), float(np.sum(v * mtw))
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.abs(mv * w).sum() * 1e-3), (lhs, rhs)
        # M differs from the identity on the replaced cells only
        assert np.abs(mv - v).max() > 0
    s.close()


def test_adjoint_window_with_weno():
    # ambient pressure 1e-4 (specific internal energy 2.5e-6 -> 2.5e-4 at
    # gamma = 1.4) and a drift of 0.002: the rarefaction at the wall the flow
    # leaves lowers the pressure by about rho c |u| = 2.4e-5, so no cell
    # reaches the 1e-6 floor (at the Sedov ambient 1e-6 and a drift of 0.02
    # the cells at that wall sit on it, where the step has no derivative);
    # random velocities of 2e-4 move every |du . n| off its kink at zero
    m, c, g, a, u, x, us = _sedov_state(drift=0.002, lift=2.475e-4, jitter=2e-4)
    n = m.ncell
    s = _solver(m, c, g, a, u, x, us)
    out = []
    for K in (1, 2):
        s.set_state(u, x, us, g, a)
        s.itime, s.dtfix, s.tacru = 7, c.dtfix, 0.0
        J, gU, gX, gS, ms = s.adjoint(2, K)
        assert np.isfinite(gU).all() and np.isfinite(gX).all() and np.isfinite(gS).all()
        out.append((J, gU, gX, gS))
    assert out[0][0] == out[1][0]
    # each schedule is bitwise repeatable; the two schedules recompute the same
    # stages but agree to rounding only (measured 1.3e-15 of the gradient scale)
    for i in (1, 2, 3):
        scale = np.abs(out[0][i]).max()
        assert np.abs(out[0][i] - out[1][i]).max() <= 1e-12 * scale, i
    # directions away from the limited region: the frozen limiter is exact there
    J0, gU = out[0][0], out[0][1]
    # the Persson marks of the window's first stage, from the oracle
    _, flags = Oracle(m, c).rhs(us.copy(), u.copy(), g.copy(), x, m.coord, a, 7)
    ctr = np.array([x[m.ipqua[i] - 1].mean(axis=0) for i in range(m.nquad)])
    # quads WENO replaces: marked, with a complete 3x3 stencil (not in the
    # boundary ring of the structured 16x16 mesh)
    ix, iy = np.arange(m.nquad) % 16, np.arange(m.nquad) // 16
    interior = (ix > 0) & (ix < 15) & (iy > 0) & (iy < 15)
    replaced = ctr[(flags[m.ntria:] > 0) & interior]
    assert len(replaced) > 0
    # at least 4 cells (h = 0.15) from every replaced quad: over the window's
    # 6 stages a perturbation there reaches no limited stencil to first order
    # in dt, so the frozen limiter's gradient is the full one
    far = np.array([np.min(np.hypot(*(replaced - p).T)) > 0.6 for p in ctr])
    assert far.sum() > 10
    rng = np.random.default_rng(5)
    eps = 1e-6
    for q in range(4):
        dvec = np.zeros((n, 4, 6))
        dvec[far, q, :] = rng.standard_normal((far.sum(), 6)) * np.abs(u[:n][far, q, :]).max()
        Jp, Jm = [], []
        for sgn, acc in ((1.0, Jp), (-1.0, Jm)):
            s.set_state(u + sgn * eps * np.concatenate([dvec, np.zeros((m.nsize - n, 4, 6))]), x, us, g, a)
            s.itime, s.dtfix, s.tacru = 7, c.dtfix, 0.0
            acc.append(s.adjoint(2, 2)[0])
        fd = (Jp[0] - Jm[0]) / (2 * eps)
        ad = float(np.sum(gU * dvec))
        assert abs(fd - ad) <= 1e-5 * max(abs(ad), 1e-12 * abs(J0)) + 1e-9 * abs(J0), (q, fd, ad)
    s.close()
