"""Run configuration of the Lag2D time step and the named benchmark workloads.

:class:`StepConfig` carries the knobs of the reference's ``module constant``
(dgflo2d.f90:4-56) that the curved-P2 time step reads.  The workloads mirror
the benchmark table: synthetic structured meshes with the sizes, gases and
initial conditions of the reference's test cases (the reference ships no
input files).
"""
from __future__ import annotations

import dataclasses
from typing import Tuple

import numpy as np

from .mesh import Mesh, hybrid_mesh, linear_quad_mesh, polar_mesh, quad_mesh

__all__ = ["StepConfig", "workload", "WORKLOADS", "noh_parity_config", "initial_density_factors"]


@dataclasses.dataclass
class StepConfig:
    npoly: int = 2
    ndegr: int = 6
    mdegr: int = 6
    nq: int = 4
    nstag: int = 3          # 2: SSP-RK2, 3: SSP-RK3 (rklag, dgflo2d.f90:320-321)
    ndt: int = 1            # 1: CFL-controlled dt (getdelt_lag), 0: fixed dtfix
    ncase: int = 1          # initial-condition / source case (getunkin)
    nlimi: int = 6
    ndens: int = 1          # first field is the specific volume tau
    ngausd: int = 7         # triangle volume rule (ctrl)
    ngausd_geo: int = 7     # triangle geometry rule (ctrl)
    gamlg: float = 1.4
    cfl: float = 0.3
    cdrho: float = 1.0      # sub-cell density correction weight
    cimpd: float = 1.0      # shock-impedance weight of the nodal solver
    tend: float = 1.0
    dtfix: float = 1.0e-4   # initial / fixed time step
    sedov_cells: Tuple[int, ...] = ()      # 1-based cells receiving the Sedov energy
    sedov_energy: float = 0.244816
    nrz: int = 0            # 0: Cartesian; RZ with y the radius on linear P1 cells: 1 true volume, 2 area-weighted

    @property
    def nmatr(self) -> int:
        return 16 if self.npoly == 2 else 4


def _tgv(n: int) -> Tuple[Mesh, StepConfig]:
    """Taylor-Green vortex at CFL 0.05: at CFL 0.1 the scheme amplifies
    perturbations of the P2 velocity moments by about 1.6x per step on meshes
    of 64x64 cells and finer (FP64, measured with the CPU restatement), at
    0.05 it does not."""
    m = quad_mesh(n, n, 0.0, 1.0, 0.0, 1.0)
    c = StepConfig(ncase=1, gamlg=5.0 / 3.0, nstag=3, cfl=0.05, tend=10.0)
    return m, c


def _sedov(n: int, cfl: float = 0.1) -> Tuple[Mesh, StepConfig]:
    """Full-box Sedov as the reference's active setup runs it
    (Getrhslagmc.f90:5634: E = 0.244816 in each of the 4 central cells);
    ``n`` x ``n`` cells on [-1.2, 1.2]^2."""
    m = quad_mesh(n, n, -1.2, 1.2, -1.2, 1.2)
    h = n // 2
    cells = ((h - 1) * n + h, (h - 1) * n + h + 1, h * n + h, h * n + h + 1)
    c = StepConfig(ncase=7, gamlg=1.4, nstag=3, cfl=cfl, tend=1.0, sedov_cells=cells)
    return m, c


def _tgv_hybrid(n: int) -> Tuple[Mesh, StepConfig]:
    """Taylor-Green on the tri/quad mesh of hybrid_mesh (alternate rows split)."""
    m = hybrid_mesh(n, n, 0.0, 1.0, 0.0, 1.0)
    c = StepConfig(ncase=1, gamlg=5.0 / 3.0, nstag=3, cfl=0.05, tend=10.0)
    return m, c


def _sedov_hybrid(n: int, jitter: float = 0.0) -> Tuple[Mesh, StepConfig]:
    """Full-box Sedov on the tri/quad mesh (alternate rows split); the energy
    goes to the first four cells (by id) that touch the centre node."""
    m = hybrid_mesh(n, n, -1.2, 1.2, -1.2, 1.2, jitter=jitter, seed=1234)
    d = np.abs(m.coord).sum(axis=1)
    centre = int(np.argmin(d)) + 1
    touch = [i + 1 for i in range(m.ntria) if centre in m.iptri[i]]
    touch += [m.ntria + i + 1 for i in range(m.nquad) if centre in m.ipqua[i]]
    c = StepConfig(ncase=7, gamlg=1.4, nstag=3, cfl=0.1, tend=1.0, sedov_cells=tuple(sorted(touch)[:4]))
    return m, c


def _noh(n: int) -> Tuple[Mesh, StepConfig]:
    """Cartesian Noh implosion (ncase 3: rho = 1, u = -r/|r|, p = 1e-6,
    gamma 5/3, SSP-RK2) on the quarter disk of polar_mesh: ``n`` rings of curved P2
    cells by ``n`` sectors, 6-node triangles on the axis ring, slip walls on
    the two rays, a free outer arc."""
    m = polar_mesh(n, n, 1.0)
    c = StepConfig(ncase=3, gamlg=5.0 / 3.0, nstag=2, cfl=0.1, tend=0.6)
    return m, c


def _sod(nx: int, ny: int, y1: float, jitter: float = 0.0) -> Tuple[Mesh, StepConfig]:
    """Sod shock tube on the linear P1 path (``ncurv = 0, nfint = 1``): straight
    4-node quads on [0,1] x [0,y1], gamma 1.4, SSP-RK2, CFL 0.3, t_end 0.2.
    The initial state follows the reference's rule, which is radial: rho = 1,
    e = 2.5 where the cell centre lies within 0.5 of the origin, rho = 0.125,
    e = 2 elsewhere (getunkin, Getrhslagmc.f90:5599-5614); slip walls all round."""
    m = linear_quad_mesh(nx, ny, 0.0, 1.0, 0.0, y1, jitter=jitter)
    c = StepConfig(npoly=1, ndegr=3, mdegr=3, ncase=6, gamlg=1.4, nstag=2, cfl=0.3, tend=0.2)
    return m, c


def _noh_square(n: int, cfl: float = 0.3) -> Tuple[Mesh, StepConfig]:
    """Cartesian Noh implosion (ncase 3, gamma 5/3, SSP-RK2) on n x n curved
    P2 quads of [0,1]^2 without triangles: slip walls on x = 0 (222) and
    y = 0 (221), free outer sides (code 22, sub-code 0).  The exact solution
    has the shock at r = t/3 with density 16 behind it, (1 + t/r) ahead."""
    m = quad_mesh(n, n, 0.0, 1.0, 0.0, 1.0)
    bf = m.bface.copy()
    for i in range(bf.shape[0]):
        if n <= i < 3 * n:          # x = 1 and y = 1: free
            bf[i, 3] = 0
    m = Mesh(coord=m.coord, ipqua=m.ipqua, iptri=m.iptri, bface=bf)
    c = StepConfig(ncase=3, gamlg=5.0 / 3.0, nstag=2, cfl=cfl, tend=0.6)
    return m, c


def _noh_rz(n: int, cfl: float = 0.3, jitter: float = 0.0, nrz: int = 1) -> Tuple[Mesh, StepConfig]:
    """Noh implosion in RZ (y is the radius, x the axial coordinate; nrz = 1
    the true-volume form, nrz = 2 the area-weighted form of
    Getrhslagrz.f90), i.e. the spherical implosion, on the
    linear P1 path: n x n straight quads on [0,1]^2, rho = 1, u = -(x, y)/r,
    p = 1e-6 (getunkin ncase 3), gamma 5/3, SSP-RK2.  x = 0 is a slip wall
    (222), y = 0 the axis (221), the outer sides are pressure boundaries
    (code 21, p = 1e-6, getbc_lagmaire2 / getbc_lagmaire_rzaw).  Node 1 is
    the origin, which the nrz = 1 node solve holds (Getrhslagmc.f90:17475);
    the area-weighted solve holds it through the two walls.  The exact
    solution has the
    shock at r = t/3 with density ((gamma+1)/(gamma-1))^3 = 64 behind it.
    ``jitter`` moves the interior vertices (seeded), for parity checks off
    the axis-aligned geometry."""
    m = linear_quad_mesh(n, n, 0.0, 1.0, 0.0, 1.0, jitter=jitter)
    bf = m.bface.copy()
    for i in range(bf.shape[0]):
        if i < n:                       # y = 0: the axis
            bf[i, 2], bf[i, 3] = 22, 221
        elif i < 3 * n:                 # x = 1 and y = 1: free, p = 1e-6
            bf[i, 2], bf[i, 3] = 21, 0
        else:                           # x = 0: slip wall
            bf[i, 2], bf[i, 3] = 22, 222
    m = Mesh(coord=m.coord, ipqua=m.ipqua, iptri=m.iptri, bface=bf, nvqua=4)
    c = StepConfig(npoly=1, ndegr=3, mdegr=3, ncase=3, gamlg=5.0 / 3.0, nstag=2, cfl=cfl, tend=0.6, nrz=nrz)
    return m, c


def initial_density_factors(mesh: Mesh, sigma: float = 0.01, seed: int = 5678) -> np.ndarray:
    """Per-cell initial-density factors 1 + sigma N(0, 1) (seeded), in cell
    order (triangles first), for lag2d_set_rho0 / Lag2DSolver.set_rho0: the
    perturbed-density Sedov setup of the hybrid-mesh adjoint case."""
    return 1.0 + sigma * np.random.default_rng(seed).standard_normal(mesh.ncell)


def noh_parity_config(c: StepConfig) -> StepConfig:
    """The Noh workload with a fixed time step of 1e-4 (ndt 0).  On this
    branch the triangles at the origin are never limited (Persson and WENO
    are quad-only) and getdelt_lag bounds dt by the sound speed and volume
    change only; from the CPU restatement, the implosion breaks down within
    a few steps at the CFL time step and by t ~ 0.02-0.06 even at fixed small
    steps, so parity runs cover the first 10 steps."""
    return dataclasses.replace(c, ndt=0, dtfix=1.0e-4)


WORKLOADS = {
    # Taylor-Green vortex: [0,1]^2, gamma 5/3, P2, RK3, energy source on
    "tgv1024": lambda: _tgv(1024),
    "tgv512": lambda: _tgv(512),
    "tgv256": lambda: _tgv(256),
    "tgv128": lambda: _tgv(128),
    "tgv64": lambda: _tgv(64),
    "tgv16": lambda: _tgv(16),
    # Sedov blast: [0,1.2]^2, gamma 1.4, energy in the corner cell
    "sedov256": lambda: _sedov(256),
    # at CFL 0.3 (the value of the reference's Sod configuration) the 32^2,
    # 64^2 and 128^2 blasts reach t = 1; at 0.1 they break down first
    "sedov32_cfl03": lambda: _sedov(32, 0.3),
    "sedov64_cfl03": lambda: _sedov(64, 0.3),
    "sedov128_cfl03": lambda: _sedov(128, 0.3),
    "sedov128": lambda: _sedov(128),
    "sedov64": lambda: _sedov(64),
    "sedov32": lambda: _sedov(32),
    "sedov16": lambda: _sedov(16),
    # the same cases on tri/quad meshes (alternate rows of quads split into triangles)
    "tgv_hybrid16": lambda: _tgv_hybrid(16),
    "tgv_hybrid64": lambda: _tgv_hybrid(64),
    "sedov_hybrid16": lambda: _sedov_hybrid(16),
    "sedov_hybrid_jitter16": lambda: _sedov_hybrid(16, jitter=0.1),
    # the adjoint case's mesh: 256x256, alternate rows split, nodes jittered by U(-0.1h, 0.1h)
    "sedov_hybrid_jitter256": lambda: _sedov_hybrid(256, jitter=0.1),
    # Noh implosion on the quarter disk (triangles on the axis ring)
    "noh100": lambda: _noh(100),
    "noh16": lambda: _noh(16),
    "noh8": lambda: _noh(8),
    # Sod on straight 4-node quads, P1 (the linear branch): the reference's 200 x 10
    # cells on [0,1] x [0,0.1], a small and a jittered case, and a 1024 x 512 one
    "sod200": lambda: _sod(200, 10, 0.1),
    "sod40": lambda: _sod(40, 4, 0.1),
    "sod_jitter40": lambda: _sod(40, 8, 0.2, jitter=0.15),
    "sod1024": lambda: _sod(1024, 512, 0.5),
    "noh_square32": lambda: _noh_square(32),
    "noh_square64": lambda: _noh_square(64),
    "noh_square100": lambda: _noh_square(100),
    "noh_rz8": lambda: _noh_rz(8),
    "noh_rz_jitter16": lambda: _noh_rz(16, jitter=0.15),
    "noh_rz32": lambda: _noh_rz(32),
    "noh_rz50": lambda: _noh_rz(50),
    "noh_rz100": lambda: _noh_rz(100),
    "noh_rz1024": lambda: _noh_rz(1024),
    "noh_rzaw8": lambda: _noh_rz(8, nrz=2),
    "noh_rzaw_jitter16": lambda: _noh_rz(16, jitter=0.15, nrz=2),
    "noh_rzaw32": lambda: _noh_rz(32, nrz=2),
    "noh_rzaw100": lambda: _noh_rz(100, nrz=2),
    "noh_rzaw1024": lambda: _noh_rz(1024, nrz=2),
}


def workload(name: str) -> Tuple[Mesh, StepConfig]:
    return WORKLOADS[name]()
