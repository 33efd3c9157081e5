"""Host-side mirror of the reference driver calls, bound to the C-ABI.

:class:`Lag2DSolver` wraps ``liblag2d.so`` (include/lag2d.h) through ctypes
with the reference's argument meanings:

* :meth:`Lag2DSolver.init_fields` -- getgeoel_initial_lag, getgeoelho_initial_lag,
  inifield_mcnew, getunkno_initial_lag (GetInitial.f90, Getrhslagmc.f90:3293);
* :meth:`Lag2DSolver.step` -- one getsolvdg_lag call plus the driver copy-back
  (Getrhslag.f90:1553, dgflo2d.f90:372-423), returning ``(dtfix, tacru)``;
* :meth:`Lag2DSolver.run` -- the driver loop (dgflo2d.f90:358-472) on the device;
* :meth:`Lag2DSolver.rhs`, :meth:`weno`, :meth:`cellvol` -- the inner seams
  getrhsdg_lag_mcnew, weno_char_quad_orthgl, getcellvol_lag.

Arrays follow the Fortran layouts (C-order numpy arrays with the Fortran
memory order): unkno ``(nsize, nq, ndegr)``, coord/ustar ``(npoin, 2)``,
geoel ``(nsize, 24)``, amatr ``(ncell, nmatr)``.  There is no CPU fallback:
loading fails with an error when the CUDA library is missing or no device is
present.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

from .config import StepConfig
from .mesh import Mesh

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBDIR = os.path.join(_HERE, "_lib")

_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)

ERRORS = {1: "EINVAL", 2: "ECUDA", 3: "EUNSUP", 4: "ENONPHYS", 5: "ESTENCIL", 6: "ENODEV"}


class Lag2DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lag2d error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class _Mesh(ctypes.Structure):
    _fields_ = [("ntria", ctypes.c_int), ("nquad", ctypes.c_int), ("npoin", ctypes.c_int),
                ("nbfac", ctypes.c_int), ("iptri", _ip), ("ipqua", _ip), ("bface", _ip),
                ("esuv1", _ip), ("esuv2", _ip), ("esqua", _ip), ("coold", _dp)]


class _Cfg(ctypes.Structure):
    _fields_ = [("npoly", ctypes.c_int), ("ndegr", ctypes.c_int), ("mdegr", ctypes.c_int),
                ("nq", ctypes.c_int), ("nstag", ctypes.c_int), ("ndt", ctypes.c_int),
                ("ncase", ctypes.c_int), ("nlimi", ctypes.c_int), ("ndens", ctypes.c_int),
                ("ngausd", ctypes.c_int), ("ngausd_geo", ctypes.c_int), ("precision", ctypes.c_int),
                ("order_exact", ctypes.c_int),
                ("nsedov", ctypes.c_int), ("sedov_cell", ctypes.c_int * 4),
                ("gamlg", ctypes.c_double), ("cfl", ctypes.c_double), ("cdrho", ctypes.c_double),
                ("cimpd", ctypes.c_double), ("tend", ctypes.c_double), ("sedov_energy", ctypes.c_double),
                ("nrz", ctypes.c_int)]


_libs = {}

EXPORTS = ("lag2d_create", "lag2d_init_fields", "lag2d_set_state", "lag2d_step", "lag2d_run",
           "lag2d_get_state", "lag2d_rhs", "lag2d_weno", "lag2d_cellvol", "lag2d_stream",
           "lag2d_kernel_launches", "lag2d_timing", "lag2d_kernel_ms", "lag2d_destroy", "lag2d_last_error",
           "lag2d_delt_noalloc", "lag2d_adjoint_step", "lag2d_adjoint", "lag2d_set_rho0",
           "lag2d_error_norms", "lag2d_weno_linear", "lag2d_cell_output")


def library_path(exact: bool = False) -> str:
    return os.path.join(_LIBDIR, "liblag2d_exact.so" if exact else "liblag2d.so")


def load(exact: bool = False):
    """Load the CUDA library (``exact``: the no-FMA parity build)."""
    key = bool(exact)
    if key in _libs:
        return _libs[key]
    path = library_path(exact)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m lag2d_b200.build`")
    lib = ctypes.CDLL(path)
    lib.lag2d_last_error.restype = ctypes.c_char_p
    lib.lag2d_kernel_launches.restype = ctypes.c_longlong
    lib.lag2d_kernel_ms.restype = ctypes.c_double
    lib.lag2d_stream.restype = ctypes.c_void_p
    lib.lag2d_stream.argtypes = [ctypes.c_void_p]
    lib.lag2d_create.argtypes = [ctypes.POINTER(_Mesh), ctypes.POINTER(_Cfg), ctypes.POINTER(ctypes.c_void_p)]
    for name in ("lag2d_init_fields", "lag2d_set_state", "lag2d_step", "lag2d_run", "lag2d_get_state",
                 "lag2d_rhs", "lag2d_weno", "lag2d_cellvol", "lag2d_timing", "lag2d_adjoint_step",
                 "lag2d_adjoint", "lag2d_set_rho0", "lag2d_error_norms", "lag2d_weno_linear",
                 "lag2d_cell_output"):
        getattr(lib, name).restype = ctypes.c_int
    lib.lag2d_destroy.argtypes = [ctypes.c_void_p]
    _libs[key] = lib
    return lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


class Lag2DSolver:
    """One mesh + configuration on the current CUDA device."""

    def __init__(self, mesh: Mesh, cfg: StepConfig, exact: bool = False, order_exact: bool = False,
                 precision: int = 0):
        """exact: load the no-FMA build; order_exact: use the kernels that keep
        the reference's summation order (both together reproduce the CPU
        restatement bit for bit); precision: 0 = FP64, 1 = FP32-mixed (bulk
        flux and quadrature arithmetic in FP32; nodal solve, node positions,
        volumes and cell-average/energy bookkeeping in FP64)."""
        self.lib = load(exact)
        self.mesh, self.cfg = mesh, cfg
        self._keep = [np.ascontiguousarray(a, dtype=np.int32) for a in
                      (mesh.iptri, mesh.ipqua, mesh.bface, mesh.esuv1, mesh.esuv2, mesh.esqua)]
        self._coold = np.ascontiguousarray(mesh.coord, dtype=np.float64)
        k = self._keep
        self._m = _Mesh(mesh.ntria, mesh.nquad, mesh.npoin, mesh.nbfac, _p(k[0], _ip), _p(k[1], _ip),
                        _p(k[2], _ip), _p(k[3], _ip), _p(k[4], _ip), _p(k[5], _ip), _p(self._coold, _dp))
        sc = (ctypes.c_int * 4)(*(list(cfg.sedov_cells) + [0, 0, 0, 0])[:4])
        self._c = _Cfg(cfg.npoly, cfg.ndegr, cfg.mdegr, cfg.nq, cfg.nstag, cfg.ndt, cfg.ncase, cfg.nlimi,
                       cfg.ndens, cfg.ngausd, cfg.ngausd_geo, int(precision), 1 if order_exact else 0,
                       len(cfg.sedov_cells),
                       sc, cfg.gamlg, cfg.cfl,
                       cfg.cdrho, cfg.cimpd, cfg.tend, cfg.sedov_energy, int(cfg.nrz))
        h = ctypes.c_void_p()
        self._check(self.lib.lag2d_create(ctypes.byref(self._m), ctypes.byref(self._c), ctypes.byref(h)))
        self.h = h
        self.dtfix = cfg.dtfix
        self.tacru = 0.0
        self.itime = 1

    def _check(self, rc: int):
        if rc != 0:
            raise Lag2DError(rc, self.lib.lag2d_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.lag2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ---------------------------------------------------------------
    def init_fields(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        m, c = self.mesh, self.cfg
        geoel = np.zeros((m.nsize, 24))
        amatr = np.zeros((m.ncell, c.nmatr))
        unkno = np.zeros((m.nsize, c.nq, c.ndegr))
        self._check(self.lib.lag2d_init_fields(self.h, _p(geoel, _dp), _p(amatr, _dp), _p(unkno, _dp)))
        self.dtfix, self.tacru, self.itime = self.cfg.dtfix, 0.0, 1
        return geoel, amatr, unkno

    def set_rho0(self, rho0):
        """Per-cell initial-density factors (ncell,) for init_fields; None
        restores the case's density."""
        a = None if rho0 is None else np.ascontiguousarray(rho0, dtype=np.float64).reshape(-1)
        if a is not None and a.size != self.mesh.ncell:
            raise ValueError("rho0 needs one value per cell")
        self._rho0 = a
        self._check(self.lib.lag2d_set_rho0(self.h, _p(a, _dp)))

    def set_state(self, unkno, coord, ustar, geoel=None, amatr=None):
        a = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None
             for x in (unkno, coord, ustar, geoel, amatr)]
        self._check(self.lib.lag2d_set_state(self.h, _p(a[0], _dp), _p(a[1], _dp), _p(a[2], _dp),
                                             _p(a[3], _dp), _p(a[4], _dp)))

    def get_state(self):
        m, c = self.mesh, self.cfg
        unkno = np.zeros((m.nsize, c.nq, c.ndegr))
        coord = np.zeros((m.npoin, 2))
        ustar = np.zeros((m.npoin, 2))
        geoel = np.zeros((m.nsize, 24))
        self._check(self.lib.lag2d_get_state(self.h, _p(unkno, _dp), _p(coord, _dp), _p(ustar, _dp),
                                             _p(geoel, _dp)))
        return unkno, coord, ustar, geoel

    # -- reference seams -------------------------------------------------------
    def step(self, itime: Optional[int] = None, dtfix: Optional[float] = None,
             tacru: Optional[float] = None) -> Tuple[float, float]:
        it = self.itime if itime is None else itime
        dt = ctypes.c_double(self.dtfix if dtfix is None else dtfix)
        ta = ctypes.c_double(self.tacru if tacru is None else tacru)
        self._check(self.lib.lag2d_step(self.h, ctypes.c_int(it), ctypes.byref(dt), ctypes.byref(ta)))
        self.dtfix, self.tacru, self.itime = dt.value, ta.value, it + 1
        return dt.value, ta.value

    def run(self, nsteps: int) -> int:
        dt = ctypes.c_double(self.dtfix)
        ta = ctypes.c_double(self.tacru)
        done = ctypes.c_int(0)
        self._check(self.lib.lag2d_run(self.h, ctypes.c_int(self.itime), ctypes.c_int(nsteps),
                                       ctypes.byref(dt), ctypes.byref(ta), ctypes.byref(done)))
        self.dtfix, self.tacru = dt.value, ta.value
        self.itime += done.value
        return done.value

    def rhs(self, itime: int = 1):
        m, c = self.mesh, self.cfg
        rhsel = np.zeros((m.ncell, c.nq, c.ndegr))
        flags = np.zeros(m.ncell, dtype=np.int32)
        self._check(self.lib.lag2d_rhs(self.h, ctypes.c_int(itime), _p(rhsel, _dp), _p(flags, _ip)))
        return rhsel, flags

    def weno(self, flags):
        f = np.ascontiguousarray(flags, dtype=np.int32)
        self._check(self.lib.lag2d_weno(self.h, _p(f, _ip)))

    def weno_linear(self, v: np.ndarray, transpose: bool = False) -> np.ndarray:
        """The WENO reconstruction at the current state with its active set
        frozen, applied to v (nsize, nq, ndegr): M(v), or M^T(v)."""
        m, c = self.mesh, self.cfg
        vin = np.zeros((m.nsize, c.nq, c.ndegr))
        vin[:v.shape[0]] = v
        out = np.zeros((m.nsize, c.nq, c.ndegr))
        self._check(self.lib.lag2d_weno_linear(self.h, ctypes.c_int(1 if transpose else 0), _p(vin, _dp),
                                               _p(out, _dp)))
        return out

    def error_norms(self) -> np.ndarray:
        """geterror_lag_curvhybrid's L2 errors of the current state against the
        exact solution: (rho, |u|, p) for Taylor-Green, (rho, e_int, p) for the
        shockless Noh case."""
        e = np.zeros(3)
        self._check(self.lib.lag2d_error_norms(self.h, _p(e, _dp)))
        return e

    def cell_output(self, badcell: bool = True):
        """End-of-run cell values from the device: (ncell, 9) array of
        (radius of the centre, rho, p, e_int, x_c, y_c, |u|, u, v) and, with
        ``badcell``, the Persson troubled-cell marker (100 or 0) per cell."""
        n = self.mesh.ncell
        out = np.zeros((n, 9))
        bad = np.zeros(n) if badcell else None
        self._check(self.lib.lag2d_cell_output(self.h, _p(out, _dp), _p(bad, _dp)))
        return out, bad

    def cellvol(self):
        geoel = np.zeros((self.mesh.nsize, 24))
        self._check(self.lib.lag2d_cellvol(self.h, _p(geoel, _dp)))
        return geoel

    # -- adjoint ---------------------------------------------------------------
    def adjoint_step(self, seed_unkno=None, seed_coord=None, seed_ustar=None, itime: Optional[int] = None):
        """One step from the handle's state plus the gradients of
        <seed, step output> w.r.t. the step input: (grad_unkno (ncell, nq,
        ndegr), grad_coord (npoin, 2), grad_ustar (npoin, 2)).  The handle
        ends at the step's output, as after step()."""
        m, c = self.mesh, self.cfg
        seeds = []
        for a, n in ((seed_unkno, m.ncell), (seed_coord, m.npoin), (seed_ustar, m.npoin)):
            seeds.append(None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.float64)[:n]))
        gu = np.zeros((m.ncell, c.nq, c.ndegr))
        gx = np.zeros((m.npoin, 2))
        gs = np.zeros((m.npoin, 2))
        it = self.itime if itime is None else itime
        dt = ctypes.c_double(self.dtfix)
        ta = ctypes.c_double(self.tacru)
        self._check(self.lib.lag2d_adjoint_step(self.h, ctypes.c_int(it), ctypes.byref(dt), ctypes.byref(ta),
                                                _p(seeds[0], _dp), _p(seeds[1], _dp), _p(seeds[2], _dp),
                                                _p(gu, _dp), _p(gx, _dp), _p(gs, _dp)))
        self.dtfix, self.tacru, self.itime = dt.value, ta.value, it + 1
        return gu, gx, gs

    def adjoint(self, nsteps: int, checkpoint_every: int):
        """nsteps steps from the handle's state and the gradient of the final
        kinetic energy J = 1/2 sum m_c (u_c^2 + v_c^2) w.r.t. the initial
        state (FP32-mixed adjoint when the solver has precision 1).  Returns (J, dJ_dunkno (ncell, nq, ndegr), dJ_dcoord (npoin, 2),
        dJ_dustar (npoin, 2), ms) with ms = [forward, recompute, reverse]
        device milliseconds."""
        m, c = self.mesh, self.cfg
        gu = np.zeros((m.ncell, c.nq, c.ndegr))
        gx = np.zeros((m.npoin, 2))
        gs = np.zeros((m.npoin, 2))
        ms = np.zeros(3)
        J = ctypes.c_double(0.0)
        dt = ctypes.c_double(self.dtfix)
        ta = ctypes.c_double(self.tacru)
        rc = self.lib.lag2d_adjoint(self.h, ctypes.c_int(self.itime), ctypes.c_int(nsteps),
                                    ctypes.c_int(checkpoint_every), ctypes.byref(dt), ctypes.byref(ta),
                                    ctypes.byref(J), _p(gu, _dp), _p(gx, _dp), _p(gs, _dp), _p(ms, _dp))
        # LAG2D_ESTENCIL (5) is a notice: a troubled quad was left unlimited, the
        # window and its gradients are complete
        self.stencil_notice = rc == 5
        if rc != 5:
            self._check(rc)
        self.dtfix, self.tacru = dt.value, ta.value
        self.itime += nsteps
        return J.value, gu, gx, gs, ms

    # -- instrumentation ---------------------------------------------------------
    @property
    def stream_ptr(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self.lib.lag2d_stream(self.h))

    def set_state_ptrs(self, unkno_ptr: int, coord_ptr: int, ustar_ptr: int):
        """set_state from raw host pointers (e.g. pinned buffers); geoel/amatr kept."""
        self._check(self.lib.lag2d_set_state(self.h, ctypes.c_void_p(unkno_ptr), ctypes.c_void_p(coord_ptr),
                                             ctypes.c_void_p(ustar_ptr), None, None))

    def get_state_ptrs(self, unkno_ptr: int, coord_ptr: int, ustar_ptr: int):
        self._check(self.lib.lag2d_get_state(self.h, ctypes.c_void_p(unkno_ptr), ctypes.c_void_p(coord_ptr),
                                             ctypes.c_void_p(ustar_ptr), None))

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.lag2d_kernel_launches(self.h))

    def timing(self, enable: bool):
        self._check(self.lib.lag2d_timing(self.h, ctypes.c_int(1 if enable else 0)))

    def kernel_ms(self, family: str):
        n = ctypes.c_longlong(0)
        ms = self.lib.lag2d_kernel_ms(self.h, family.encode(), ctypes.byref(n))
        return (ms if ms >= 0 else None), int(n.value)
