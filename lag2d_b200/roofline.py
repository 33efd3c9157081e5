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
(its inputs read once, its outputs written once), so the intermediate arrays
the split into kernels introduces (corner coefficients, the RHS) are counted
where they are written and where they are read.
"""
from __future__ import annotations

W = 8  # FP64 bytes


def stage_bytes(ncell: int, npoin: int, ndegr: int = 6, nq: int = 4) -> int:
    return ncell * (3 * ndegr * nq * W + 16 * W + 5 * W + 8 + 9 * 4) + npoin * (4 * 16 + 2 * 16 + 4) + 16 * ncell * 4


def kernel_bytes(family: str, ncell: int, npoin: int) -> int:
    """Interface bytes of one launch of a kernel family on an all-quad mesh."""
    U = 24 * W            # 24 DOFs of one cell
    GEO = 5 * W           # rc, sc, g19..g21
    CONN = 9 * 4          # ipqua row
    CF = 160 * W          # corner coefficients of one quad (5 values x 32 corner faces)
    XY = 2 * W
    fam = {
        # U, geometry, sub-cell masses, connectivity, nodes (x, ustar) -> corner coefficients
        "corner": ncell * (U + GEO + 4 * W + CONN + CF) + npoin * (XY + XY),
        # corner coefficients via the gather list + ustar in/out + masks -> ustar
        "node": ncell * (CF + 32 * 4) + npoin * (4 + 1 + XY + XY),
        # U, geometry, connectivity, corner coefficients, nodes (x, ustar) -> RHS
        "rhs": ncell * (U + GEO + CONN + CF + U) + npoin * (XY + XY),
        # RHS, U^n, U^(s) in/out, M^-1
        "update": ncell * (U + U + 2 * U + 16 * W),
        # U, geometry, mass, connectivity, x, X0 -> flag, physical centre, frame
        "persson": ncell * (U + GEO + W + CONN + 4 + 2 * W + 4 * W) + npoin * (XY + XY),
        "nodes": npoin * (XY + XY + XY + XY),
        "geom": ncell * (CONN + 3 * W) + npoin * XY,
    }
    return fam[family]
