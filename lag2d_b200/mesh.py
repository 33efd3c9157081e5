"""Mesh and control-file handling for the Lag2D time step.

Covers what the reference driver reads before its time loop:

* ``dgflo2d.ctrl`` (13 value lines, Preprocess.f90:28-55) -> :class:`Ctrl`;
* ``dgflo2d.domn`` (Preprocess.f90:156-220, 605-660) -> :class:`Mesh`;
* the derived connectivity the step uses: the cells-surrounding-point CSR
  ``esuv1/esuv2`` (Preprocess.f90:719-790) and the quad face neighbours
  ``esqua`` (getesuel, dgflo2d.f90:1220-1309; boundary faces carry the ghost
  id ``ncell + iface``).

It also generates the structured 9-node quadrilateral meshes the benchmark
workloads use (Sod, Sedov, Taylor-Green), numbered the way a mesh file for the
reference would be: cells row by row, the nine nodes of a quad ordered
corners (counter-clockwise from (-1,-1)), edge mid-nodes, centre.

All integer arrays hold 1-based ids, as in the Fortran arrays; a 2-D array
``a`` of shape ``(n, k)`` in C order has the memory layout of the Fortran
array ``a(k, n)``.
"""
from __future__ import annotations

import dataclasses
import io
import os
from typing import Optional

import numpy as np

__all__ = ["Mesh", "Ctrl", "quad_mesh", "hybrid_mesh", "polar_mesh", "read_domn", "write_domn", "read_ctrl", "write_ctrl",
           "build_esuv", "build_esqua"]


@dataclasses.dataclass
class Mesh:
    """Mesh arrays in the reference's conventions (1-based ids)."""
    coord: np.ndarray            # (npoin, 2) float64  == coord(2, npoin)
    ipqua: np.ndarray            # (nquad, 9) int32    == ipqua(9, nquad)
    iptri: np.ndarray            # (ntria, 6) int32    == iptri(6, ntria)
    bface: np.ndarray            # (nbfac, 5) int32    == bface(5, nbfac)
    esuv1: np.ndarray = None     # (npoin1,) int32
    esuv2: np.ndarray = None     # (npoin+1,) int32
    esqua: np.ndarray = None     # (nquad, 4) int32    == esqua(4, nquad)
    nvqua: int = 9               # nodes per quad: 9 (curved, ncurv=1) or 4 (straight, ncurv=0)

    def __post_init__(self):
        self.coord = np.ascontiguousarray(self.coord, dtype=np.float64)
        self.ipqua = np.ascontiguousarray(self.ipqua, dtype=np.int32).reshape(-1, self.nvqua)
        self.iptri = np.ascontiguousarray(self.iptri, dtype=np.int32).reshape(-1, 6)
        self.bface = np.ascontiguousarray(self.bface, dtype=np.int32).reshape(-1, 5)
        if self.esuv1 is None or self.esuv2 is None:
            self.esuv1, self.esuv2 = build_esuv(self.iptri, self.ipqua, self.npoin)
        if self.esqua is None:
            self.esqua = build_esqua(self.ipqua, self.iptri, self.bface)

    @property
    def ntria(self) -> int:
        return int(self.iptri.shape[0])

    @property
    def nquad(self) -> int:
        return int(self.ipqua.shape[0])

    @property
    def npoin(self) -> int:
        return int(self.coord.shape[0])

    @property
    def nbfac(self) -> int:
        return int(self.bface.shape[0])

    @property
    def ncell(self) -> int:
        return self.ntria + self.nquad

    @property
    def nsize(self) -> int:
        return self.ncell + self.nbfac


@dataclasses.dataclass
class Ctrl:
    """The values of ``dgflo2d.ctrl`` (Preprocess.f90:28-55)."""
    amach: float = 0.0
    cfl: float = 0.3
    nflux: int = 1
    breta: float = 0.0
    dtfix: float = 1.0e-4
    nmatel: int = 1
    gamlg: float = 1.4
    cdrho: float = 1.0
    tend: float = 1.0
    cimpd: float = 1.0
    ntime: int = 100
    ndegr: int = 6
    mdegr: int = 6
    npoly: int = 2
    nreco: int = 0
    nlimi: int = 6
    ngaus: int = 3
    ngausf: int = 3
    ngausd: int = 7
    nint: int = 1
    ngausf_geo: int = 3
    ngausd_geo: int = 7
    ncurv: int = 1
    nresi: int = 1
    nmeth: int = 2
    nq: int = 4
    ndens: int = 1
    ndt: int = 1
    nstag: int = 3
    ncase: int = 1
    nriem: int = 1
    nfint: int = 4
    nrz: int = 0
    nout: int = 0
    ndump: int = 0

    _LINES = (("amach", "cfl", "nflux", "breta", "dtfix"), ("nmatel",),
              ("gamlg", "cdrho", "tend", "cimpd"), ("ntime", "ndegr", "mdegr", "npoly", "nreco"),
              ("nlimi", "ngaus", "ngausf", "ngausd", "nint"), ("ngausf_geo", "ngausd_geo"),
              ("ncurv",), ("nresi",), ("nmeth", "nq", "ndens"), ("ndt", "nstag"),
              ("ncase", "nriem", "nfint"), ("nrz",), ("nout", "ndump"))


def _fortran_float(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "e"))


def read_ctrl(path_or_text: str) -> Ctrl:
    """Parse a ``dgflo2d.ctrl``: a comment line before each of the 13 value lines."""
    text = open(path_or_text).read() if os.path.exists(path_or_text) else path_or_text
    lines = text.splitlines()
    c = Ctrl()
    for k, names in enumerate(Ctrl._LINES):
        toks = lines[2 * k + 1].replace(",", " ").split()
        for name, tok in zip(names, toks):
            cur = getattr(c, name)
            setattr(c, name, int(float(tok)) if isinstance(cur, int) else _fortran_float(tok))
    return c


def write_ctrl(c: Ctrl, path: Optional[str] = None) -> str:
    out = io.StringIO()
    for names in Ctrl._LINES:
        out.write("  " + " ".join(names) + "\n")
        vals = []
        for n in names:
            v = getattr(c, n)
            vals.append(repr(float(v)).replace("e", "d") if isinstance(v, float) else str(v))
        out.write("  " + " ".join(vals) + "\n")
    s = out.getvalue()
    if path:
        with open(path, "w") as f:
            f.write(s)
    return s


def read_domn(path: str) -> Mesh:
    """Parse a ``dgflo2d.domn`` as preprocess1/preprocess2 read it (curved, nvqua=9, nvtri=6)."""
    with open(path) as f:
        lines = f.read().splitlines()
    pos = 0
    nn = int(lines[pos].split()[0]); pos += 1 + nn
    pos += 1  # title
    ndimn, ntype = (int(t) for t in lines[pos].split()[:2]); pos += 1
    pos += 1
    hdr = lines[pos].replace("d", "e").split(); pos += 1
    ntria, npoin, nbfac, nquad = int(hdr[0]), int(hdr[1]), int(hdr[2]), int(hdr[4])
    pos += 1
    iptri = np.array([[int(t) for t in lines[pos + i].split()[1:7]] for i in range(ntria)],
                     dtype=np.int32).reshape(-1, 6); pos += ntria
    ipqua = np.array([[int(t) for t in lines[pos + i].split()[1:10]] for i in range(nquad)],
                     dtype=np.int32).reshape(-1, 9); pos += nquad
    pos += 1
    coord = np.array([[_fortran_float(t) for t in lines[pos + i].split()[1:3]] for i in range(npoin)],
                     dtype=np.float64); pos += npoin
    pos += 1 + npoin  # unused per-point block
    pos += 1
    bface = np.array([[int(t) for t in lines[pos + i].split()[1:6]] for i in range(nbfac)],
                     dtype=np.int32).reshape(-1, 5)
    return Mesh(coord=coord, ipqua=ipqua, iptri=iptri, bface=bface)


def write_domn(m: Mesh, path: str) -> None:
    with open(path, "w") as f:
        f.write("1\n generated by lag2d_b200.mesh\n")
        f.write(" mesh\n 2 1\n ntria npoin nbfac tinpt nquad\n")
        f.write(f" {m.ntria} {m.npoin} {m.nbfac} 0.0 {m.nquad}\n")
        f.write(" connectivity\n")
        for i, row in enumerate(m.iptri):
            f.write(f"{i + 1} " + " ".join(str(int(v)) for v in row) + "\n")
        for i, row in enumerate(m.ipqua):
            f.write(f"{i + 1} " + " ".join(str(int(v)) for v in row) + "\n")
        f.write(" coordinates\n")
        for i, (x, y) in enumerate(m.coord):
            f.write(f"{i + 1} {float(x)!r} {float(y)!r}\n")
        f.write(" unknowns\n")
        for i in range(m.npoin):
            f.write(f"{i + 1} 0.0 0.0 0.0 0.0\n")
        f.write(" boundary faces\n")
        for i, row in enumerate(m.bface):
            f.write(f"{i + 1} " + " ".join(str(int(v)) for v in row) + "\n")


def build_esuv(iptri: np.ndarray, ipqua: np.ndarray, npoin: int):
    """Cells surrounding each point, CSR with ``esuv2[0] = 0`` (Preprocess.f90:719-790).

    Triangles are numbered first, then quads (ielem = ntria + iquad); each
    point's list is in increasing cell order because cells are visited in order.
    """
    ntria = iptri.shape[0]
    cells = np.concatenate([np.repeat(np.arange(1, ntria + 1, dtype=np.int64), iptri.shape[1]),
                            np.repeat(np.arange(ntria + 1, ntria + ipqua.shape[0] + 1, dtype=np.int64),
                                      ipqua.shape[1])])
    pts = np.concatenate([iptri.reshape(-1).astype(np.int64), ipqua.reshape(-1).astype(np.int64)])
    order = np.lexsort((cells, pts))
    counts = np.bincount(pts - 1, minlength=npoin)
    esuv2 = np.zeros(npoin + 1, dtype=np.int32)
    esuv2[1:] = np.cumsum(counts)
    esuv1 = cells[order].astype(np.int32)
    return esuv1, esuv2


def boundary_hosts(iptri: np.ndarray, ipqua: np.ndarray, bface: np.ndarray) -> np.ndarray:
    """Host cell of each boundary face (1-based, triangles first), the
    result of preprocess1's step 2 (Preprocess.f90:679-717).

    The reference tests every cell's corner vertices against both end points
    of every boundary face, O(nbfac x ncell), and keeps the last cell that
    holds both (triangles, then quads).  Here every pair of corner vertices
    of every cell is keyed once and the boundary faces are looked up in the
    sorted keys: O((ncell + nbfac) log ncell), same answer (0 where no cell
    holds both end points)."""
    ntria, nquad = iptri.shape[0], ipqua.shape[0]
    pairs, cells = [], []
    for conn, nv, first in ((iptri, 3, 1), (ipqua, 4, ntria + 1)):
        if conn.shape[0] == 0:
            continue
        corner = conn[:, :nv].astype(np.int64)
        ids = np.arange(first, first + conn.shape[0], dtype=np.int64)
        for a in range(nv):
            for b in range(a + 1, nv):
                lo = np.minimum(corner[:, a], corner[:, b])
                hi = np.maximum(corner[:, a], corner[:, b])
                pairs.append(lo * (1 << 32) + hi)
                cells.append(ids)
    hosts = np.zeros(bface.shape[0], dtype=np.int32)
    if not pairs or bface.shape[0] == 0:
        return hosts
    keys = np.concatenate(pairs)
    owner = np.concatenate(cells)
    order = np.lexsort((owner, keys))       # by key, then cell id: the last of a run is the highest id
    ks, os_ = keys[order], owner[order]
    last = np.ones(ks.size, dtype=bool)
    last[:-1] = ks[1:] != ks[:-1]
    ks, os_ = ks[last], os_[last]
    b0 = bface[:, 0].astype(np.int64)
    b1 = bface[:, 1].astype(np.int64)
    q = np.minimum(b0, b1) * (1 << 32) + np.maximum(b0, b1)
    pos = np.searchsorted(ks, q)
    pos = np.minimum(pos, ks.size - 1)
    hit = ks[pos] == q
    hosts[hit] = os_[pos[hit]].astype(np.int32)
    return hosts


def build_esqua(ipqua: np.ndarray, iptri: np.ndarray, bface: np.ndarray) -> np.ndarray:
    """Cell across each quad face (face k joins corner k and corner k+1).

    Interior faces get the neighbouring cell id, boundary faces the ghost id
    ``ncell + iface`` as getesuel assigns through intfac (dgflo2d.f90:1220-1309).
    """
    ntria, nquad = iptri.shape[0], ipqua.shape[0]
    ncell = ntria + nquad
    edge_owner = {}
    for t in range(ntria):
        v = iptri[t, :3]
        for k in range(3):
            a, b = int(v[k]), int(v[(k + 1) % 3])
            edge_owner.setdefault((min(a, b), max(a, b)), []).append(t + 1)
    corners = ipqua[:, :4].astype(np.int64)
    a = corners
    b = np.roll(corners, -1, axis=1)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    keys = lo * (int(ipqua.max()) + 1) + hi
    flat = keys.reshape(-1)
    order = np.argsort(flat, kind="stable")
    sk = flat[order]
    esqua = np.zeros((nquad, 4), dtype=np.int32)
    same = np.nonzero(sk[1:] == sk[:-1])[0]
    f1, f2 = order[same], order[same + 1]
    esqua[f1 // 4, f1 % 4] = f2 // 4 + ntria + 1
    esqua[f2 // 4, f2 % 4] = f1 // 4 + ntria + 1
    if ntria:
        for q in range(nquad):
            for k in range(4):
                if esqua[q, k] == 0:
                    key = (int(lo[q, k]), int(hi[q, k]))
                    if key in edge_owner:
                        esqua[q, k] = edge_owner[key][0]
    bkey = {}
    for i, row in enumerate(bface):
        x, y = int(row[0]), int(row[1])
        bkey[(min(x, y), max(x, y))] = i + 1
    qs, ks = np.nonzero(esqua == 0)
    for q, k in zip(qs.tolist(), ks.tolist()):
        key = (int(lo[q, k]), int(hi[q, k]))
        esqua[q, k] = ncell + bkey[key] if key in bkey else 0
    return esqua


def quad_mesh(nx: int, ny: int, x0: float = 0.0, x1: float = 1.0, y0: float = 0.0, y1: float = 1.0,
              jitter: float = 0.0, curve: float = 0.0, seed: int = 1234,
              wall_code: int = 22) -> Mesh:
    """Structured ``nx`` x ``ny`` mesh of 9-node quads on ``[x0,x1] x [y0,y1]``.

    ``jitter`` moves interior vertices by U(-jitter*h, jitter*h) (seeded);
    ``curve`` moves interior edge mid-nodes normal-ish by U(-curve*h, curve*h),
    which curves the cell edges.  The centre node is placed where the step's
    re-interpolation puts it (-1/4 of the corners + 1/2 of the edge nodes,
    Getrhslag.f90:1963-1971).  Boundary faces are slip walls: ``bface(3) =
    wall_code`` with sub-code 221 on the y-walls (v fixed) and 222 on the
    x-walls (u fixed), as getndvelo_lagsubg applies them.
    """
    nxl, nyl = 2 * nx + 1, 2 * ny + 1
    hx, hy = (x1 - x0) / nx, (y1 - y0) / ny
    ii, jj = np.meshgrid(np.arange(nxl), np.arange(nyl))  # jj rows
    X = x0 + ii * (hx / 2.0)
    Y = y0 + jj * (hy / 2.0)
    rng = np.random.default_rng(seed)
    if jitter > 0.0:
        vi, vj = np.meshgrid(np.arange(2, nxl - 2, 2), np.arange(2, nyl - 2, 2))
        X[vj, vi] += rng.uniform(-jitter * hx, jitter * hx, size=vi.shape)
        Y[vj, vi] += rng.uniform(-jitter * hy, jitter * hy, size=vi.shape)
    # edge mid-nodes at the midpoint of their end vertices
    X[:, 1::2] = 0.5 * (X[:, 0:-1:2] + X[:, 2::2])
    Y[:, 1::2] = 0.5 * (Y[:, 0:-1:2] + Y[:, 2::2])
    X[1::2, :] = 0.5 * (X[0:-1:2, :] + X[2::2, :])
    Y[1::2, :] = 0.5 * (Y[0:-1:2, :] + Y[2::2, :])
    if curve > 0.0:
        # horizontal edge mids (even row, odd col) move in y; vertical (odd row, even col) in x
        hr, hc = np.meshgrid(np.arange(1, nxl - 1, 2), np.arange(2, nyl - 2, 2))
        Y[hc, hr] += rng.uniform(-curve * hy, curve * hy, size=hr.shape)
        vr, vc = np.meshgrid(np.arange(2, nxl - 2, 2), np.arange(1, nyl - 1, 2))
        X[vc, vr] += rng.uniform(-curve * hx, curve * hx, size=vr.shape)
    nid = (jj * nxl + ii + 1).astype(np.int64)
    ci, cj = np.meshgrid(np.arange(nx), np.arange(ny))
    ci, cj = ci.reshape(-1), cj.reshape(-1)

    def at(di, dj):
        return nid[2 * cj + dj, 2 * ci + di]

    ipqua = np.stack([at(0, 0), at(2, 0), at(2, 2), at(0, 2),
                      at(1, 0), at(2, 1), at(1, 2), at(0, 1), at(1, 1)], axis=1).astype(np.int32)
    coord = np.stack([X.reshape(-1), Y.reshape(-1)], axis=1)
    c = ipqua - 1
    for d in range(2):
        v = coord[:, d]
        v[c[:, 8]] = -0.25 * (v[c[:, 0]] + v[c[:, 1]] + v[c[:, 2]] + v[c[:, 3]]) + \
            0.5 * (v[c[:, 4]] + v[c[:, 5]] + v[c[:, 6]] + v[c[:, 7]])
    bf = []
    for i in range(nx):  # bottom: corner1 -> corner2 of cell (i, 0)
        bf.append((nid[0, 2 * i], nid[0, 2 * i + 2], wall_code, 221, nid[0, 2 * i + 1]))
    for j in range(ny):  # right
        bf.append((nid[2 * j, nxl - 1], nid[2 * j + 2, nxl - 1], wall_code, 222, nid[2 * j + 1, nxl - 1]))
    for i in range(nx - 1, -1, -1):  # top
        bf.append((nid[nyl - 1, 2 * i + 2], nid[nyl - 1, 2 * i], wall_code, 221, nid[nyl - 1, 2 * i + 1]))
    for j in range(ny - 1, -1, -1):  # left
        bf.append((nid[2 * j + 2, 0], nid[2 * j, 0], wall_code, 222, nid[2 * j + 1, 0]))
    bface = np.array(bf, dtype=np.int32)
    return Mesh(coord=coord, ipqua=ipqua, iptri=np.zeros((0, 6), np.int32), bface=bface)


def hybrid_mesh(nx: int, ny: int, x0: float = 0.0, x1: float = 1.0, y0: float = 0.0, y1: float = 1.0,
                jitter: float = 0.0, curve: float = 0.0, seed: int = 1234, split_rows=None,
                wall_code: int = 22) -> Mesh:
    """Curved tri/quad mesh: the structured 9-node quad mesh of :func:`quad_mesh`
    with the quads of alternate rows (``j % 2 == 1`` unless ``split_rows`` is
    given) split along the diagonal from corner 1 to corner 3 into two 6-node
    triangles (nodes: 3 vertices counter-clockwise, then the mid-nodes of
    edges 1-2, 2-3 and 3-1).  The quad's centre node becomes the mid-node of
    the diagonal and is moved to its midpoint.  Triangles are numbered first,
    as the reference numbers them (ielem = itria, then ntria + iquad).
    """
    q = quad_mesh(nx, ny, x0, x1, y0, y1, jitter=jitter, curve=curve, seed=seed, wall_code=wall_code)
    rows = set(range(1, ny, 2)) if split_rows is None else set(split_rows)
    coord = q.coord.copy()
    tris, quads = [], []
    for c in range(q.nquad):
        j = c // nx
        n = q.ipqua[c]
        if j in rows:
            a, b, cc, d, eab, ebc, ecd, eda, m = (int(v) for v in n)
            coord[m - 1] = 0.5 * (coord[a - 1] + coord[cc - 1])
            tris.append((a, b, cc, eab, ebc, m))
            tris.append((a, cc, d, m, ecd, eda))
        else:
            quads.append(tuple(int(v) for v in n))
    # the unsplit quads keep the centre-node rule of the step (quad_mesh placed it so)
    return Mesh(coord=coord, ipqua=np.array(quads, dtype=np.int32).reshape(-1, 9),
                iptri=np.array(tris, dtype=np.int32).reshape(-1, 6), bface=q.bface)


def polar_mesh(nr: int, nt: int, radius: float = 1.0, wall_code: int = 22) -> Mesh:
    """Quarter disk ``0 <= theta <= pi/2``, ``r <= radius`` of ``nr`` rings by
    ``nt`` sectors with curved (P2) cells: the innermost ring is 6-node
    triangles meeting at the origin, the others 9-node quads.  Nodes lie on
    the exact circles and rays (edge mid-nodes at mid-radius or mid-angle);
    the quad centre node is placed by the step's re-interpolation rule.
    Boundary faces: the ray theta = 0 is a slip wall with v fixed
    (``bface(3) = wall_code``, sub-code 221), the ray theta = pi/2 one with u
    fixed (sub-code 222), the outer arc is free (sub-code 0).  Triangles are
    numbered first, cells ring by ring.
    """
    dr, dt = radius / nr, 0.5 * np.pi / nt
    ids = {}
    xy = []

    def node(a, b):
        """Node at half-step lattice point (radius a dr/2, angle b dt/2); a = 0 is the origin."""
        key = (0, 0) if a == 0 else (a, b)
        if key not in ids:
            ids[key] = len(xy) + 1
            r, t = 0.5 * a * dr, 0.5 * b * dt
            xy.append((r * np.cos(t), r * np.sin(t)))
        return ids[key]

    tris, quads = [], []
    for j in range(nt):
        b0, b1, b2 = 2 * j, 2 * j + 1, 2 * j + 2
        tris.append((node(0, 0), node(2, b0), node(2, b2), node(1, b0), node(2, b1), node(1, b2)))
    for i in range(1, nr):
        a0, a1, a2 = 2 * i, 2 * i + 1, 2 * i + 2
        for j in range(nt):
            b0, b1, b2 = 2 * j, 2 * j + 1, 2 * j + 2
            quads.append((node(a0, b0), node(a2, b0), node(a2, b2), node(a0, b2),
                          node(a1, b0), node(a2, b1), node(a1, b2), node(a0, b1), node(a1, b1)))
    coord = np.array(xy, dtype=np.float64)
    ipqua = np.array(quads, dtype=np.int32).reshape(-1, 9)
    c = ipqua - 1
    for d in range(2):
        v = coord[:, d]
        v[c[:, 8]] = -0.25 * (v[c[:, 0]] + v[c[:, 1]] + v[c[:, 2]] + v[c[:, 3]]) + \
            0.5 * (v[c[:, 4]] + v[c[:, 5]] + v[c[:, 6]] + v[c[:, 7]])
    bf = []
    # theta = 0: origin outwards (domain on the left)
    bf.append((node(0, 0), node(2, 0), wall_code, 221, node(1, 0)))
    for i in range(1, nr):
        bf.append((node(2 * i, 0), node(2 * i + 2, 0), wall_code, 221, node(2 * i + 1, 0)))
    # outer arc, counter-clockwise
    for j in range(nt):
        bf.append((node(2 * nr, 2 * j), node(2 * nr, 2 * j + 2), wall_code, 0, node(2 * nr, 2 * j + 1)))
    # theta = pi/2: inwards to the origin
    for i in range(nr - 1, 0, -1):
        bf.append((node(2 * i + 2, 2 * nt), node(2 * i, 2 * nt), wall_code, 222, node(2 * i + 1, 2 * nt)))
    bf.append((node(2, 2 * nt), node(0, 0), wall_code, 222, node(1, 2 * nt)))
    return Mesh(coord=coord, ipqua=ipqua, iptri=np.array(tris, dtype=np.int32).reshape(-1, 6),
                bface=np.array(bf, dtype=np.int32))


def linear_quad_mesh(nx: int, ny: int, x0: float = 0.0, x1: float = 1.0, y0: float = 0.0,
                     y1: float = 1.0, jitter: float = 0.0, seed: int = 1234,
                     wall_code: int = 22) -> Mesh:
    """Structured ``nx`` x ``ny`` mesh of straight 4-node quads (``ncurv = 0``,
    ``ipqua(4, nquad)``) on ``[x0,x1] x [y0,y1]``, counter-clockwise corners,
    cells row by row.  ``jitter`` moves interior vertices by U(-jitter*h,
    jitter*h) (seeded).  Boundary faces as in :func:`quad_mesh` (slip walls,
    221 on the y-walls, 222 on the x-walls; the mid-node column is 0).
    """
    hx, hy = (x1 - x0) / nx, (y1 - y0) / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1))
    X = x0 + ii * hx
    Y = y0 + jj * hy
    X[:, nx] = x1
    Y[ny, :] = y1
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        vi, vj = np.meshgrid(np.arange(1, nx), np.arange(1, ny))
        X[vj, vi] += rng.uniform(-jitter * hx, jitter * hx, size=vi.shape)
        Y[vj, vi] += rng.uniform(-jitter * hy, jitter * hy, size=vi.shape)
    nid = (jj * (nx + 1) + ii + 1).astype(np.int64)
    ci, cj = np.meshgrid(np.arange(nx), np.arange(ny))
    ci, cj = ci.reshape(-1), cj.reshape(-1)
    ipqua = np.stack([nid[cj, ci], nid[cj, ci + 1], nid[cj + 1, ci + 1], nid[cj + 1, ci]],
                     axis=1).astype(np.int32)
    coord = np.stack([X.reshape(-1), Y.reshape(-1)], axis=1)
    bf = []
    for i in range(nx):
        bf.append((nid[0, i], nid[0, i + 1], wall_code, 221, 0))
    for j in range(ny):
        bf.append((nid[j, nx], nid[j + 1, nx], wall_code, 222, 0))
    for i in range(nx - 1, -1, -1):
        bf.append((nid[ny, i + 1], nid[ny, i], wall_code, 221, 0))
    for j in range(ny - 1, -1, -1):
        bf.append((nid[j + 1, 0], nid[j, 0], wall_code, 222, 0))
    return Mesh(coord=coord, ipqua=ipqua, iptri=np.zeros((0, 3), np.int32),
                bface=np.array(bf, dtype=np.int32), nvqua=4)
