"""Run a few time steps of a named workload, for profilers (ncu) and quick checks.

    python -m lag2d_b200.profile_step tgv256 2            # FP64 step
    python -m lag2d_b200.profile_step tgv256 2 --mixed    # FP32-mixed step
    python -m lag2d_b200.profile_step tgv256 2 --adjoint 1  # lag2d_adjoint over 2 steps

Each step is one lag2d_step call (no graph), so every kernel launch of the
step is visible to a profiler in launch order.
"""
from __future__ import annotations

import argparse

from .api import Lag2DSolver
from .config import initial_density_factors, workload


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", nargs="?", default="tgv256")
    ap.add_argument("steps", nargs="?", type=int, default=2)
    ap.add_argument("--mixed", action="store_true", help="FP32-mixed form (precision = 1)")
    ap.add_argument("--rho0", action="store_true",
                    help="per-cell initial densities 1 + 0.01 N(0, 1) (seed 5678) before the initial fields")
    ap.add_argument("--adjoint", type=int, default=0, metavar="K",
                    help="run lag2d_adjoint over the steps with checkpoints every K steps")
    a = ap.parse_args()
    m, c = workload(a.workload)
    s = Lag2DSolver(m, c, precision=1 if a.mixed else 0)
    if a.rho0:
        s.set_rho0(initial_density_factors(m))
    s.init_fields()
    if a.adjoint > 0:
        J, _, _, _, ms = s.adjoint(a.steps, a.adjoint)
        print(f"adjoint J={J:.12e} forward/recompute/reverse ms = {ms[0]:.3f} {ms[1]:.3f} {ms[2]:.3f}")
    else:
        for _ in range(a.steps):
            s.step()
    print(f"ok {a.workload} steps={a.steps} mixed={a.mixed} dtfix={s.dtfix:.6e} tacru={s.tacru:.6e}")
    s.close()


if __name__ == "__main__":
    main()
