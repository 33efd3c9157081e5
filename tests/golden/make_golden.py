"""Regenerates the oracle fixtures in this folder.

The reference (Fortran) cannot be compiled in this environment and ships no
golden outputs, so these fixtures pin the CPU oracle against regressions and
give the GPU path fixed targets: small Taylor-Green and Sedov runs (8 x 8, a
12 x 12 Sedov with troubled cells, a curved 6 x 6 quad mesh, a curved
tri/quad mesh and the Noh implosion on a 4 x 4 quarter-disk mesh with
triangles at the origin), 3 time steps each, and the radial Sod problem on a
jittered 12 x 4 mesh of straight quads on the linear P1 path, 6 steps; and the
Sedov problem on 32 x 32 quads run to t_end = 1 (`sedov32_tend`: cell averages
and coordinates only).

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py tgv6_hybrid # one fixture
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lag2d_b200 import quad_mesh, StepConfig  # noqa: E402
from lag2d_b200.mesh import hybrid_mesh, linear_quad_mesh, polar_mesh  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

CASES = {
    "tgv8": (lambda: quad_mesh(8, 8, 0.0, 1.0, 0.0, 1.0),
             StepConfig(ncase=1, gamlg=5.0 / 3.0, nstag=3, cfl=0.1, tend=10.0), 3),
    "sedov12": (lambda: quad_mesh(12, 12, -1.2, 1.2, -1.2, 1.2),
                StepConfig(ncase=7, gamlg=1.4, nstag=3, cfl=0.1, tend=1.0, sedov_cells=(66, 67, 78, 79)), 3),
    "tgv6_curved": (lambda: quad_mesh(6, 6, 0.0, 1.0, 0.0, 1.0, jitter=0.1, curve=0.05, seed=7),
                    StepConfig(ncase=1, gamlg=5.0 / 3.0, nstag=2, cfl=0.1, tend=10.0), 3),
    # curved tri/quad mesh (alternate rows split into 6-node triangles)
    "tgv6_hybrid": (lambda: hybrid_mesh(6, 6, 0.0, 1.0, 0.0, 1.0, jitter=0.1, curve=0.05, seed=7),
                    StepConfig(ncase=1, gamlg=5.0 / 3.0, nstag=3, cfl=0.05, tend=10.0), 3),
    # Noh on the curved quarter disk, fixed time step
    "noh4_polar": (lambda: polar_mesh(4, 4),
                   StepConfig(ncase=3, gamlg=5.0 / 3.0, nstag=3, ndt=0, dtfix=1.0e-4, tend=0.6), 3),
    # radial Sod on jittered straight quads, linear P1 branch (ncurv=0, nfint=1)
    "sod12_p1": (lambda: linear_quad_mesh(12, 4, 0.0, 1.0, 0.0, 0.4, jitter=0.15, seed=7),
                 StepConfig(npoly=1, ndegr=3, mdegr=3, ncase=6, gamlg=1.4, nstag=2, cfl=0.3, tend=0.2), 6),
}


def run_case(name):
    mk, cfg, nsteps = CASES[name]
    m = mk()
    o = Oracle(m, cfg)
    geoel, amatr, unkno = o.init()
    u0, g0 = unkno.copy(), geoel.copy()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    _, dt, ta = o.run(unkno, coord, m.coord, geoel, amatr, ustar, 1, nsteps, cfg.dtfix, 0.0)
    return dict(unkno0=u0, geoel0=g0, geoel=geoel, amatr=amatr, unkno=unkno, coord=coord, ustar=ustar,
                dtfix=np.float64(dt), tacru=np.float64(ta), nsteps=np.int64(nsteps))


def run_to_end(name="sedov32"):
    """The full-box Sedov problem on 32 x 32 quads run to t_end = 1 (322
    steps): cell averages, coordinates and the driver scalars only."""
    from lag2d_b200.config import workload
    m, c = workload(name)
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    n, dt, ta = o.run(unkno, coord, m.coord, geoel, amatr, ustar, 1, 1000, c.dtfix, 0.0)
    return dict(avg=unkno[:m.ncell, :, 0].copy(), coord=coord, dtfix=np.float64(dt), tacru=np.float64(ta),
                nsteps=np.int64(n))


if __name__ == "__main__":
    for name in (sys.argv[1:] or list(CASES) + ["sedov32_tend"]):
        data = run_to_end() if name == "sedov32_tend" else run_case(name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print("wrote", name)
