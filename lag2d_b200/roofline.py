"""Compulsory (algorithmic) HBM bytes of the time step and of each kernel family.

Stage level (the whole RK stage, each input read once and each output
written once, intermediates excluded), FP64:

    B_stage = N_c * (3*ndegr*nq*8 + 16*8 + 5*8 + 8 + 9*4)
            + N_p * (4*16 + 2*16 + 4) + 16*N_c*4

  3*ndegr*nq*8  read U^n and U^(s), write U^(s+1)
  16*8          M^-1 (amatr)
  5*8           reference mass centre rc, sc and the P2 offsets g19..g21
  8             the cell volume written
  9*4           connectivity of a 9-node quad
  per node      read x^n, x^(s), X_0, ustar_prev (4 x 16 B); write x^(s+1),
                ustar (2 x 16 B); a CSR offset (4 B)
  16*N_c*4      the node-to-corner gather list (16 corners per quad)

Per kernel family the same rule is applied to that kernel's own interface
(its inputs read once, its outputs written once), for the optimised kernels
the step runs (the RHS pass takes the face integral from the corner pass's
node partial sums):

  corner   U^(s), rc/sc/g19..g21, sub-cell masses, connectivity, x^(s),
           ustar_prev -> 4 sub-cell corrections, 45 node partial sums
  node     45 partial sums and 9 gather ids per quad, CSR offset, mask,
           ustar_prev -> ustar
  dt       (stage 1) connectivity, cell averages, volume, x^(s), ustar
           -> two per-block minima
  rhs      U^(s), U^n, M^-1, geometry, the 40 partial sums of the 8
           boundary nodes, connectivity, x^(s), ustar (+ the 6 source
           moments on Taylor-Green) -> U^(s+1) (the M^-1 solve and RK
           combine are fused into every stage)
  src      (Taylor-Green) connectivity, geometry, x^(s) -> 6 source moments
  persson  tau DOFs, mean velocity, geometry, mass, shape moments,
           connectivity, x^(s) -> flag, physical centre, frame
  nodes    x^n, x^(s), ustar -> x^(s+1), ustar_prev
  geom     connectivity, x^(s) -> volume, centre node
"""
from __future__ import annotations

W = 8  # FP64 bytes


def stage_bytes(ncell: int, npoin: int, ndegr: int = 6, nq: int = 4) -> int:
    return ncell * (3 * ndegr * nq * W + 16 * W + 5 * W + 8 + 9 * 4) + npoin * (4 * 16 + 2 * 16 + 4) + 16 * ncell * 4


def stage_bytes_p1(ncell: int, npoin: int) -> int:
    """The same stage rule on the linear P1 path (straight 4-node quads):
    12 DOFs per cell, M^-1 of 4 values, rc/sc, the volume, 4 node ids, the
    same node traffic, 4 corners per quad in the node-to-corner list."""
    return ncell * (3 * 3 * 4 * W + 4 * W + 2 * W + 8 + 4 * 4) + npoin * (4 * 16 + 2 * 16 + 4) + 4 * ncell * 4


def kernel_bytes(family: str, ncell: int, npoin: int, nstag: int = 3, source: bool = False) -> int:
    """Interface bytes of one launch of a kernel family on an all-quad mesh,
    averaged over the family's launches in one time step (``source``: the
    Taylor-Green source moments are read by the RHS pass)."""
    U = 24 * W            # 24 DOFs of one cell
    GEO = 5 * W           # rc, sc, g19..g21
    CONN = 9 * 4          # ipqua row
    XY = 2 * W            # one node pair (x, y) or (u, v)
    fam = {
        "corner": ncell * (U + GEO + 4 * W + CONN + 4 * W + 45 * W) + npoin * (XY + XY),
        "node": ncell * (45 * W + 9 * 4) + npoin * (4 + 1 + XY + XY),
        "dt": ncell * (CONN + 4 * W + W) + npoin * 2 * XY,
        "rhs": ncell * (U + U + 16 * W + GEO + 40 * W + CONN + U + (6 * W if source else 0)) + npoin * 2 * XY,
        "src": ncell * (CONN + GEO + 6 * W) + npoin * XY,
        "persson": ncell * (6 * W + 2 * W + GEO + W + 9 * W + CONN + 4 + 2 * W + 4 * W) + npoin * XY,
        "nodes": npoin * (3 * XY + 2 * XY),
        "geom": ncell * (CONN + W + XY) + npoin * XY,
    }
    return fam[family]
