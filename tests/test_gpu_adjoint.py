"""Adjoint of the optimised FP64 step (lag2d_adjoint, lag2d_adjoint_step).

The functional is the final kinetic energy J = 1/2 sum_c m_c (u_c^2 + v_c^2)
after 3 RK3 steps with a fixed time step (ndt = 0) with the Taylor-Green
source and a randomly perturbed initial state (every DOF moves, so no
symmetry line leaves a kink of |du.n| at zero), on a curved, jittered 8x8
quad mesh and on a curved, jittered 6x6 tri/quad mesh (alternate rows split
into 6-node triangles).

Bounds:
  * directional derivatives <dJ/dU, d> and <dJ/dx, d> against central finite
    differences of the same GPU step, (J(+eps d) - J(-eps d)) / (2 eps) with
    eps = 1e-5, within 1e-5 relative plus the differences' round-off floor
    4 u J / eps (u = 2^-53);
  * the gradients do not depend on the checkpoint interval (bit for bit: the
    recomputed segments repeat the forward arithmetic exactly), and the handle
    ends at the same state as plain steps;
  * a torch.autograd.Function around lag2d_step / lag2d_adjoint_step, chained
    over the 3 steps, gives the gradients of the checkpointed window to 1e-12;
  * the FP32-mixed adjoint (precision 1: mixed forward passes, FP32
    volume-integral and sub-cell-mass transposes) gives every directional
    derivative of the FP64 adjoint to MIXED_TOL relative (or of the largest
    one, for derivatives near zero);
  * configurations outside the differentiated path (order_exact) report LAG2D_EUNSUP.
"""
import dataclasses

import numpy as np
import pytest
import torch

from lag2d_b200 import StepConfig, quad_mesh, workload
from lag2d_b200.mesh import hybrid_mesh
from lag2d_b200.api import Lag2DError, Lag2DSolver

pytestmark = pytest.mark.gpu

NSTEPS = 3
EPS = 1e-5
FD_TOL = 1e-5
MIXED_TOL = 1e-4


def _case(kind):
    if kind == "quad":
        m = quad_mesh(8, 8, jitter=0.1, curve=0.08, seed=4)
    else:
        m = hybrid_mesh(6, 6, jitter=0.1, curve=0.05, seed=7)
    c = StepConfig(ncase=1, gamlg=5.0 / 3.0, nstag=3, cfl=0.05, tend=10.0, ndt=0)
    s = Lag2DSolver(m, c)
    geoel, amatr, unkno = s.init_fields()
    n = m.ncell
    rng = np.random.default_rng(7)
    for q in range(4):
        sc = max(np.abs(unkno[:n, q, 0]).max(), 1e-2)
        unkno[:n, q, 0] += 1e-2 * sc * rng.standard_normal(n) * (0.2 if q == 0 else 1.0)
        unkno[:n, q, 1:3] += 1e-3 * sc * rng.standard_normal((n, 2))
        unkno[:n, q, 3:] += 1e-4 * sc * rng.standard_normal((n, 3))
    return m, c, s, geoel, amatr, unkno


def _reset(s, c, unkno, coord, ustar, geoel=None, amatr=None):
    s.set_state(unkno, coord, ustar, geoel, amatr)
    s.itime, s.dtfix, s.tacru = 1, c.dtfix, 0.0


def _energy(s, mass):
    u = s.get_state()[0]
    n = mass.size
    return 0.5 * np.sum(mass * (u[:n, 1, 0] ** 2 + u[:n, 2, 0] ** 2))


@pytest.fixture(scope="module", params=["quad", "hybrid"])
def case(request):
    m, c, s, geoel, amatr, unkno = _case(request.param)
    zero = np.zeros_like(m.coord)
    _reset(s, c, unkno, m.coord, zero, geoel, amatr)
    J, gU, gX, gS, ms = s.adjoint(NSTEPS, 2)
    return dict(m=m, c=c, s=s, geoel=geoel, amatr=amatr, unkno=unkno, J=J, gU=gU, gX=gX, gS=gS, ms=ms)


def test_adjoint_matches_finite_differences(case):
    m, c, s, unkno = case["m"], case["c"], case["s"], case["unkno"]
    gU, gX, J = case["gU"], case["gX"], case["J"]
    n = m.ncell
    mass = case["geoel"][:n, 3].copy()
    zero = np.zeros_like(m.coord)

    def J_of(u, x):
        _reset(s, c, u, x, zero)
        for _ in range(NSTEPS):
            s.step()
        return _energy(s, mass)

    assert abs(J_of(unkno, m.coord) - J) <= 1e-14 * J
    floor = 4 * 2.0 ** -53 * J / EPS
    rng = np.random.default_rng(11)
    dx = 1.0 / np.sqrt(n)
    checked = 0
    for q in range(4):
        for kk, order in (([0], 0), ([1, 2], 1), ([3, 4, 5], 2)):
            d = np.zeros_like(unkno)
            scale = max(np.abs(unkno[:n, q, 0]).max(), 1e-2) * dx ** order
            for k in kk:
                d[:n, q, k] = rng.standard_normal(n) * scale
            fd = (J_of(unkno + EPS * d, m.coord) - J_of(unkno - EPS * d, m.coord)) / (2 * EPS)
            ad = float(np.sum(gU * d[:n]))
            assert abs(fd - ad) <= FD_TOL * abs(ad) + floor, (q, kk, fd, ad)
            checked += 1
    for _ in range(3):
        d = rng.standard_normal(m.coord.shape) * dx * 0.1
        fd = (J_of(unkno, m.coord + EPS * d) - J_of(unkno, m.coord - EPS * d)) / (2 * EPS)
        ad = float(np.sum(gX * d))
        assert abs(fd - ad) <= FD_TOL * abs(ad) + floor, ("coord", fd, ad)
        checked += 1
    assert checked == 15


def test_adjoint_ustar_gradient(case):
    """The previous nodal velocity enters the first stage's impedance."""
    m, c, s, unkno = case["m"], case["c"], case["s"], case["unkno"]
    n = m.ncell
    mass = case["geoel"][:n, 3].copy()
    rng = np.random.default_rng(5)
    d = rng.standard_normal(m.coord.shape) * 1e-2

    def J_of(us):
        _reset(s, c, unkno, m.coord, us)
        for _ in range(NSTEPS):
            s.step()
        return _energy(s, mass)

    zero = np.zeros_like(m.coord)
    fd = (J_of(zero + EPS * d) - J_of(zero - EPS * d)) / (2 * EPS)
    ad = float(np.sum(case["gS"] * d))
    floor = 4 * 2.0 ** -53 * case["J"] / EPS
    assert abs(fd - ad) <= FD_TOL * abs(ad) + floor, (fd, ad)


def test_checkpoint_interval_invariance(case):
    m, c, s, unkno = case["m"], case["c"], case["s"], case["unkno"]
    zero = np.zeros_like(m.coord)
    _reset(s, c, unkno, m.coord, zero)
    for _ in range(NSTEPS):
        s.step()
    u_ref, x_ref, us_ref, _ = s.get_state()
    for K in (1, NSTEPS, 7):
        _reset(s, c, unkno, m.coord, zero)
        J, gU, gX, gS, ms = s.adjoint(NSTEPS, K)
        assert J == case["J"]
        assert np.array_equal(gU, case["gU"]) and np.array_equal(gX, case["gX"]) and np.array_equal(gS, case["gS"])
        u, x, us, _ = s.get_state()
        assert np.array_equal(u[:m.ncell], u_ref[:m.ncell]) and np.array_equal(x, x_ref) and np.array_equal(us, us_ref)
        assert (ms > 0).all()


class _Step(torch.autograd.Function):
    """One lag2d_step as a differentiable map (unkno, coord, ustar) -> same,
    with lag2d_adjoint_step as its backward (test harness only)."""

    @staticmethod
    def forward(ctx, solver, itime, base, unkno, coord, ustar):
        ctx.solver, ctx.itime, ctx.base = solver, itime, base
        ctx.save_for_backward(unkno, coord, ustar)
        c = solver.cfg
        full = base.copy()
        full[:unkno.shape[0]] = unkno.detach().numpy()
        _reset(solver, c, full, coord.detach().numpy(), ustar.detach().numpy())
        solver.step(itime=itime)
        u, x, us, _ = solver.get_state()
        return torch.from_numpy(u[:unkno.shape[0]].copy()), torch.from_numpy(x), torch.from_numpy(us)

    @staticmethod
    def backward(ctx, gu, gx, gs):
        unkno, coord, ustar = ctx.saved_tensors
        solver = ctx.solver
        full = ctx.base.copy()
        full[:unkno.shape[0]] = unkno.detach().numpy()
        _reset(solver, solver.cfg, full, coord.detach().numpy(), ustar.detach().numpy())
        su, sx, ss = (None if g is None else g.detach().contiguous().numpy() for g in (gu, gx, gs))
        a, b, d = solver.adjoint_step(su, sx, ss, itime=ctx.itime)
        return None, None, None, torch.from_numpy(a), torch.from_numpy(b), torch.from_numpy(d)


def test_autograd_function_chain(case):
    m, s, unkno = case["m"], case["s"], case["unkno"]
    n = m.ncell
    mass = torch.from_numpy(case["geoel"][:n, 3].copy())
    u0 = torch.from_numpy(unkno[:n].copy()).requires_grad_(True)
    x0 = torch.from_numpy(m.coord.copy()).requires_grad_(True)
    s0 = torch.zeros_like(x0).requires_grad_(True)
    u, x, us = u0, x0, s0
    for it in range(1, NSTEPS + 1):
        u, x, us = _Step.apply(s, it, unkno, u, x, us)
    J = 0.5 * torch.sum(mass * (u[:, 1, 0] ** 2 + u[:, 2, 0] ** 2))
    J.backward()
    assert abs(J.item() - case["J"]) <= 1e-14 * case["J"]
    for got, ref in ((u0.grad.numpy(), case["gU"]), (x0.grad.numpy(), case["gX"]), (s0.grad.numpy(), case["gS"])):
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_adjoint_hybrid_sedov_window():
    """Sedov on the jittered tri/quad mesh with per-cell initial densities
    1 + 0.01 N(0, 1): the Persson sensor marks quads,
    but WENO replaces none (every quad's 3x3 stencil reaches a triangle), so
    a 2-step window is differentiable; its gradients are finite and do not
    depend on the checkpoint interval."""
    from lag2d_b200.config import initial_density_factors
    m, c = workload("sedov_hybrid_jitter16")
    s = Lag2DSolver(m, dataclasses.replace(c, ndt=0))
    s.set_rho0(initial_density_factors(m))
    g, a, u = s.init_fields()
    out = []
    for K in (1, 2):
        _reset(s, s.cfg, u, m.coord, np.zeros_like(m.coord), g, a)
        J, gU, gX, gS, ms = s.adjoint(2, K)
        assert np.isfinite(gU).all() and np.isfinite(gX).all() and np.isfinite(gS).all()
        out.append((J, gU, gX))
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])


def test_adjoint_unsupported_configurations():
    m, c = workload("tgv16")
    s = Lag2DSolver(m, c, order_exact=True)
    s.init_fields()
    with pytest.raises(Lag2DError) as e:
        s.adjoint_step()
    assert e.value.code == 3


def test_mixed_adjoint_against_fp64_adjoint(case):
    m, c, unkno = case["m"], case["c"], case["unkno"]
    n = m.ncell
    sm = Lag2DSolver(m, c, precision=1)
    sm.init_fields()
    _reset(sm, c, unkno, m.coord, np.zeros_like(m.coord), case["geoel"], case["amatr"])
    J, gU, gX, gS, ms = sm.adjoint(NSTEPS, 2)
    assert abs(J - case["J"]) <= 1e-6 * case["J"]
    rng = np.random.default_rng(3)
    dirs = []
    for q in range(4):
        for kk in ([0], [1, 2], [3, 4, 5]):
            d = np.zeros((n, 4, 6))
            for k in kk:
                d[:, q, k] = rng.standard_normal(n)
            dirs.append((float(np.sum(gU * d)), float(np.sum(case["gU"] * d)), f"U q={q} k={kk}"))
    for _ in range(3):
        d = rng.standard_normal(m.coord.shape)
        dirs.append((float(np.sum(gX * d)), float(np.sum(case["gX"] * d)), "coord"))
        dirs.append((float(np.sum(gS * d)), float(np.sum(case["gS"] * d)), "ustar"))
    big = max(abs(r) for _, r, _ in dirs)
    for got, ref, what in dirs:
        assert abs(got - ref) <= MIXED_TOL * max(abs(ref), 1e-3 * big), (what, got, ref)
