"""Run a named workload through the driver loop to its end time (or a number
of steps) on the device and report what the reference's own run would print
or write: steps, final time, conservation of mass and total energy, and for
the radial cases (Noh, Sod, Sedov) the radius of the density peak of the cell
averages (the shock position), for Taylor-Green the L2 errors.

    python -m lag2d_b200.run_case sedov128            # to t_end = 1
    python -m lag2d_b200.run_case tgv256 --steps 200
    python -m lag2d_b200.run_case sod1024 --steps 100

The loop is lag2d_run in chunks (dgflo2d.f90:358-472 on the device, exit
test at t_end included).  Two modes for profilers (ncu) replace the chunked
loop, so that every kernel launch of a step is visible in launch order:

    python -m lag2d_b200.run_case tgv256 --steps 2 --per-step          # one lag2d_step per step, no graph
    python -m lag2d_b200.run_case tgv256 --steps 2 --per-step --mixed  # the FP32-mixed step
    python -m lag2d_b200.run_case tgv256 --steps 2 --adjoint 1         # lag2d_adjoint over 2 steps, K = 1
"""
from __future__ import annotations

import argparse
import ctypes
import dataclasses
import time

import numpy as np

from .api import Lag2DError, Lag2DSolver
from .config import initial_density_factors, workload

LAG2D_ESTENCIL = 5


def run_chunk(s: Lag2DSolver, nsteps: int):
    """lag2d_run for nsteps; LAG2D_ESTENCIL (a troubled quad whose vertex
    valence the reference's WENO stops on, left unlimited) is reported, not
    raised: the steps were completed."""
    dt, ta, done = ctypes.c_double(s.dtfix), ctypes.c_double(s.tacru), ctypes.c_int(0)
    rc = s.lib.lag2d_run(s.h, ctypes.c_int(s.itime), ctypes.c_int(nsteps), ctypes.byref(dt), ctypes.byref(ta),
                         ctypes.byref(done))
    if rc not in (0, LAG2D_ESTENCIL):
        raise Lag2DError(rc, s.lib.lag2d_last_error().decode())
    s.dtfix, s.tacru = dt.value, ta.value
    s.itime += done.value
    return done.value, rc == LAG2D_ESTENCIL


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload")
    ap.add_argument("--steps", type=int, default=0, help="stop after this many steps (0: run to t_end)")
    ap.add_argument("--chunk", type=int, default=500)
    ap.add_argument("--mixed", action="store_true", help="FP32-mixed form (precision = 1)")
    ap.add_argument("--cfl", type=float, default=0.0, help="override the workload's CFL number")
    ap.add_argument("--rho0", action="store_true",
                    help="per-cell initial densities 1 + 0.01 N(0, 1) (seed 5678) before the initial fields")
    ap.add_argument("--per-step", action="store_true",
                    help="one lag2d_step call per step (no graph), for profilers; prints one line")
    ap.add_argument("--adjoint", type=int, default=0, metavar="K",
                    help="run lag2d_adjoint over --steps steps with checkpoints every K steps; prints one line")
    a = ap.parse_args()
    m, c = workload(a.workload)
    if a.cfl > 0:
        c = dataclasses.replace(c, cfl=a.cfl)
    s = Lag2DSolver(m, c, precision=1 if a.mixed else 0)
    if a.rho0:
        s.set_rho0(initial_density_factors(m))
    geoel, _, unkno = s.init_fields()
    if a.per_step or a.adjoint > 0:
        nsteps = max(a.steps, 1)
        if a.adjoint > 0:
            J, _, _, _, ms = s.adjoint(nsteps, a.adjoint)
            print(f"adjoint J={J:.12e} forward/recompute/reverse ms = {ms[0]:.3f} {ms[1]:.3f} {ms[2]:.3f}")
        else:
            for _ in range(nsteps):
                s.step()
        print(f"ok {a.workload} steps={nsteps} mixed={a.mixed} dtfix={s.dtfix:.6e} tacru={s.tacru:.6e}")
        s.close()
        return
    n = m.ncell
    mass = geoel[:n, 3].copy()
    e0 = float((mass * unkno[:n, 3, 0]).sum())
    limit = a.steps if a.steps > 0 else 10 ** 9
    done, stencil, t0 = 0, 0, time.perf_counter()
    while done < limit:
        k, st = run_chunk(s, min(a.chunk, limit - done))
        done += k
        stencil += int(st)
        if k == 0 or abs(s.tacru - c.tend) <= 1e-11 * c.tend:
            break
    wall = time.perf_counter() - t0
    u, x, _, g = s.get_state()
    e1 = float((mass * u[:n, 3, 0]).sum())
    print(f"{a.workload}: {done} steps to t = {s.tacru:.6g} (t_end {c.tend:g}), last dt {s.dtfix:.3e}, "
          f"{1e3 * wall / max(done, 1):.3f} ms per step (wall, chunks of {a.chunk})")
    if stencil:
        print(f"  {stencil} chunk(s) reported LAG2D_ESTENCIL: troubled quads at a vertex valence the "
              "reference's WENO stops on (WENO.f90:7699) were left unlimited")
    print(f"  cell masses unchanged: {bool(np.array_equal(g[:n, 3], mass))}; "
          f"total energy of the cell averages: relative change {(e1 - e0) / e0:.3e}; "
          f"min volume {g[:n, 2].min():.3e}")
    if c.ncase in (3, 6, 7):
        rho = g[:n, 3] / g[:n, 2]
        quads = x[m.ipqua[:, :4] - 1]
        ctr = quads.mean(axis=1)
        r = np.hypot(ctr[:, 0], ctr[:, 1])
        top = np.argsort(rho)[-max(4, n // 1000):]
        print(f"  density peak {rho.max():.4f} at radius {r[int(np.argmax(rho))]:.4f}; "
              f"mean radius of the densest 0.1% of cells {r[top].mean():.4f}")
    if c.ncase in (1, 2) and m.ntria == 0 and c.npoly == 2:
        e = s.error_norms()
        print(f"  L2 errors (rho, |u|, p): {e[0]:.3e} {e[1]:.3e} {e[2]:.3e}")
    s.close()


if __name__ == "__main__":
    main()
