"""End-of-run output of the Lagrangian driver: restart files, the cell VTK
file and the radial profile file, in the reference's formats.

The per-cell values come from the device (``Lag2DSolver.cell_output``,
C-ABI ``lag2d_cell_output``); this module only formats them.

* ``write_restart`` / ``read_restart``: ``restartdg.dat`` as the driver
  writes it at the end of a run (dgflo2d.f90:489-496: per cell, the ndegr
  moments of each of the 4 fields with the Fortran format ``(3e32.16)``),
  plus ``restartlag.dat``, which the reference does not write: the time
  state (itime, tacru, dtfix) and per node the coordinates and the nodal
  velocity u*, without which a Lagrangian run cannot continue (the
  reference's own restart reader is disabled for the Lagrangian method,
  Getrhslagmc.f90:3922-3937).
* ``write_vtk``: ``output.vtk`` of getoutput_cellvtk (Postprocess.f90:1258-1398):
  points, cells (VTK types 5/9 for ncurv = 0, 22/23 for ncurv = 1), and the
  cell data density, internal energy, pressure, Badcell and velocity.
* ``write_profile``: the per-cell radial profile file of the error routine,
  ``unradicurv.dat`` (geterror_lag_curvhybrid, Postprocess.f90:3700-3717,
  :3944-3983) or ``unradi.dat`` on straight cells (geterror_lag_hybrid,
  :3515-3582), for the cases the reference writes it for.
"""
import math
from typing import Optional, Tuple

import numpy as np


def fortran_e(x: float, w: int, d: int) -> str:
    """Fortran ``Ew.d`` edit descriptor: 0.ddd...E+xx right-justified in w."""
    x = float(x)
    if x != x:
        return "NaN".rjust(w)
    if x == 0.0:
        mant, exp = "0." + "0" * d, 0
        s = f"{mant}E+00"
    else:
        # round to d significant digits, then write as 0.ddd x 10^exp
        m = f"{abs(x):.{d - 1}e}"
        digits, e10 = m.split("e")
        exp = int(e10) + 1
        s = "0." + digits.replace(".", "") + ("E+" if exp >= 0 else "E-") + f"{abs(exp):02d}"
        if x < 0:
            s = "-" + s
        return s.rjust(w)
    return s.rjust(w)


def _fortran_lines(values, per_line: int, w: int, d: int):
    """Format reversion of ``(n ew.d)``: per_line values per record."""
    vals = list(values)
    out = []
    for i in range(0, len(vals), per_line):
        out.append("".join(fortran_e(v, w, d) for v in vals[i:i + per_line]))
    return out


# ---------------------------------------------------------------------------
# restart
# ---------------------------------------------------------------------------
def write_restart(directory: str, unkno: np.ndarray, coord: np.ndarray, ustar: np.ndarray,
                  itime: int, tacru: float, dtfix: float, ncell: Optional[int] = None,
                  centre: Optional[np.ndarray] = None) -> Tuple[str, str]:
    """Write restartdg.dat (reference format) and restartlag.dat (coordinates,
    nodal velocities and time state) into ``directory``; ``unkno`` is
    (nsize or ncell, nq, ndegr) as Lag2DSolver.get_state returns it.
    ``centre`` (ncell, 2), geoel(1:2) of get_state, is appended to
    restartlag.dat when given: the area-weighted RZ form (nrz = 2) moves the
    mass centre every stage and its limiter reads it before renewing it."""
    import os
    u = np.asarray(unkno, dtype=np.float64)
    n = u.shape[0] if ncell is None else ncell
    p1 = os.path.join(directory, "restartdg.dat")
    with open(p1, "w") as f:
        for e in range(n):
            for q in range(u.shape[1]):
                f.write("\n".join(_fortran_lines(u[e, q], 3, 32, 16)) + "\n")
    p2 = os.path.join(directory, "restartlag.dat")
    x = np.asarray(coord, dtype=np.float64)
    s = np.asarray(ustar, dtype=np.float64)
    with open(p2, "w") as f:
        f.write(f"{int(itime)} {float(tacru)!r} {float(dtfix)!r} {x.shape[0]}\n")
        for i in range(x.shape[0]):
            f.write(f"{float(x[i, 0])!r} {float(x[i, 1])!r} {float(s[i, 0])!r} {float(s[i, 1])!r}\n")
        if centre is not None:
            cen = np.asarray(centre, dtype=np.float64)
            f.write(f"{cen.shape[0]}\n")
            for e in range(cen.shape[0]):
                f.write(f"{float(cen[e, 0])!r} {float(cen[e, 1])!r}\n")
    return p1, p2


def read_restart(directory: str, ncell: int, nq: int = 4, ndegr: int = 6, with_centre: bool = False):
    """Read the pair write_restart wrote: (unkno (ncell, nq, ndegr), coord
    (npoin, 2), ustar (npoin, 2), itime, tacru, dtfix), and with
    ``with_centre`` the mass centres (ncell, 2) or None if the file has
    none.  restartdg.dat keeps 16 significant digits, as the reference
    writes it; restartlag.dat is exact."""
    import os
    with open(os.path.join(directory, "restartdg.dat")) as f:
        vals = np.array([float(t.replace("D", "E")) for t in f.read().split()])
    if vals.size != ncell * nq * ndegr:
        raise ValueError(f"restartdg.dat holds {vals.size} values, expected {ncell * nq * ndegr}")
    unkno = vals.reshape(ncell, nq, ndegr)
    with open(os.path.join(directory, "restartlag.dat")) as f:
        head = f.readline().split()
        itime, tacru, dtfix, npoin = int(head[0]), float(head[1]), float(head[2]), int(head[3])
        rows = np.array([[float(t) for t in f.readline().split()] for _ in range(npoin)])
        head = f.readline().split()
        centre = None
        if head:
            centre = np.array([[float(t) for t in f.readline().split()] for _ in range(int(head[0]))])
    out = (unkno, rows[:, :2].copy(), rows[:, 2:4].copy(), itime, tacru, dtfix)
    return out + (centre,) if with_centre else out


# ---------------------------------------------------------------------------
# VTK cell file
# ---------------------------------------------------------------------------
def write_vtk(path: str, mesh, coord: np.ndarray, cellout: np.ndarray, badcell: Optional[np.ndarray],
              ncurv: int = 1) -> None:
    """getoutput_cellvtk: ``cellout`` (ncell, 9) from Lag2DSolver.cell_output
    (radius, rho, p, e_int, x_c, y_c, |u|, u, v), ``badcell`` the Persson
    marker per cell (zeros if None).  The internal energy is p / rho /
    (gamma - 1), equal to the reference's e - (u^2 + v^2)/2 up to rounding."""
    x = np.asarray(coord, dtype=np.float64)
    nt, nqd, nc = mesh.ntria, mesh.nquad, mesh.ncell
    nvtri, nvqua = mesh.iptri.shape[1], mesh.ipqua.shape[1]
    mtype = (5, 9) if ncurv == 0 else (22, 23)
    bad = np.zeros(nc) if badcell is None else np.asarray(badcell, dtype=np.float64)
    lines = ["# vtk DataFile Version 2.0", "Unstructured Grid Example", "ASCII", "",
             "DATASET UNSTRUCTURED_GRID", f" Points {x.shape[0]}  float "]
    lines += [f" {float(x[i, 0])!r} {float(x[i, 1])!r} 0.0" for i in range(x.shape[0])]
    lines += ["", f" CELLS {nc} {(nvtri + 1) * nt + (nvqua + 1) * nqd}"]
    lines += ["".join(f"{v:10d}" for v in [nvtri, *(mesh.iptri[i] - 1)]) for i in range(nt)]
    lines += ["".join(f"{v:10d}" for v in [nvqua, *(mesh.ipqua[i] - 1)]) for i in range(nqd)]
    lines += ["", f" CELL_TYPES {nc}"]
    lines += [f" {mtype[0]}"] * nt + [f" {mtype[1]}"] * nqd
    lines += ["", "", f" CELL_DATA {nc}", " SCALARS density float", " LOOKUP_TABLE default"]
    lines += [f" {float(v)!r}" for v in cellout[:, 1]]
    lines += ["", " SCALARS internalenergy float", " LOOKUP_TABLE default"]
    lines += [fortran_e(v, 20, 8) for v in cellout[:, 3]]
    lines += ["", " SCALARS pressure float", " LOOKUP_TABLE default"]
    lines += [fortran_e(v, 20, 8) for v in cellout[:, 2]]
    lines += ["", " SCALARS Badcell float", " LOOKUP_TABLE default"]
    lines += [fortran_e(v, 20, 8) for v in bad]
    lines += ["", " VECTORS vectors float"]
    lines += [fortran_e(cellout[e, 7], 32, 16) + fortran_e(cellout[e, 8], 32, 16) + fortran_e(0.0, 32, 16)
              for e in range(nc)]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_vtk_cell_data(path: str) -> dict:
    """The CELL_DATA scalars and vectors of a file write_vtk wrote (for checks)."""
    with open(path) as f:
        toks = f.read().split("\n")
    out, i = {}, 0
    nc = None
    while i < len(toks):
        t = toks[i].split()
        if t[:1] == ["CELL_DATA"]:
            nc = int(t[1])
        elif t[:1] == ["SCALARS"] and nc is not None:
            name = t[1]
            out[name] = np.array([float(toks[i + 2 + k]) for k in range(nc)])
            i += 2 + nc
            continue
        elif t[:1] == ["VECTORS"] and nc is not None:
            out[t[1]] = np.array([[float(v) for v in toks[i + 1 + k].split()] for k in range(nc)])
            i += 1 + nc
            continue
        i += 1
    return out


# ---------------------------------------------------------------------------
# radial profile file
# ---------------------------------------------------------------------------
def profile_lines(mesh, cellout: np.ndarray, ncase: int, curved: bool = True):
    """The records the error routine writes to its profile file, one per cell
    (triangles first): ``(i8, 9e32.16)`` ielem, r, rho, p, e_int, x_c, y_c,
    |u|, u, v for quads in the shock cases; the other layouts as the
    routine selects them by ncase.  No records for the smooth cases (1, 2)."""
    recs = []
    fmt = lambda ielem, vals: f"{ielem:8d}" + "".join(fortran_e(v, 32, 16) for v in vals)
    nt = mesh.ntria
    c = cellout
    if curved:
        if ncase in (7, 6, 3, 8):
            for e in range(nt):
                r, rho, p, ei, xc, yc, um, u, v = c[e]
                recs.append(fmt(e + 1, (r, rho, p, ei) if ncase == 6 else (r, rho, p, ei, um, u, v)))
        if ncase in (7, 6, 3, 4, 8, 12, 13, 15):
            for e in range(nt, mesh.ncell):
                r, rho, p, ei, xc, yc, um, u, v = c[e]
                if ncase in (6, 7, 3, 4, 10, 11, 14, 8):
                    recs.append(fmt(e + 1, (r, rho, p, ei, xc, yc, um, u, v)))
                if ncase in (12, 13, 15):
                    recs.append(fmt(e + 1, (xc, rho, p, ei, um, u, v)))
    else:
        if ncase in (7, 6, 3, 4, 8, 10, 11, 12, 13, 14):
            for e in range(nt, mesh.ncell):
                r, rho, p, ei, xc, yc, um, u, v = c[e]
                if ncase in (6, 7, 8, 3, 4, 10, 11, 14):
                    recs.append(fmt(e + 1, (r, rho, p, ei, xc, yc, um, u, v)))
                if ncase == 12:
                    recs.append(fmt(e + 1, (xc, rho, p, ei, um, u, v)))
                if ncase == 13:
                    recs.append(fmt(e + 1, (math.sqrt(xc * xc), rho, p, ei, xc, yc, u, v)))
    return recs


def write_profile(directory: str, mesh, cellout: np.ndarray, ncase: int, curved: bool = True) -> str:
    import os
    path = os.path.join(directory, "unradicurv.dat" if curved else "unradi.dat")
    with open(path, "w") as f:
        recs = profile_lines(mesh, cellout, ncase, curved)
        f.write("\n".join(recs) + ("\n" if recs else ""))
    return path


def shock_radius(cellout: np.ndarray) -> Tuple[float, float]:
    """(radius, density) of the densest cell: the shock position the profile
    file is read for in the Sedov and Noh problems."""
    i = int(np.argmax(cellout[:, 1]))
    return float(cellout[i, 0]), float(cellout[i, 1])
