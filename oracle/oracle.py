"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/_build/liblag2d_oracle.so`` (built by ``make -C oracle``) and
exposes the restated reference routines on numpy arrays.  Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liblag2d_oracle.so")
_lib = None

_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


class _OMesh(ctypes.Structure):
    _fields_ = [("ntria", ctypes.c_int), ("nquad", ctypes.c_int), ("npoin", ctypes.c_int),
                ("nbfac", ctypes.c_int), ("iptri", _ip), ("ipqua", _ip), ("bface", _ip),
                ("esuv1", _ip), ("esuv2", _ip), ("esqua", _ip), ("nvqua", ctypes.c_int)]


class _OCfg(ctypes.Structure):
    _fields_ = [("npoly", ctypes.c_int), ("ndegr", ctypes.c_int), ("mdegr", ctypes.c_int),
                ("nq", ctypes.c_int), ("nstag", ctypes.c_int), ("ndt", ctypes.c_int),
                ("ncase", ctypes.c_int), ("nlimi", ctypes.c_int), ("ndens", ctypes.c_int),
                ("ngausd", ctypes.c_int), ("ngausd_geo", ctypes.c_int),
                ("sedov_ncell", ctypes.c_int), ("sedov_cell", ctypes.c_int * 4),
                ("gamlg", ctypes.c_double), ("cfl", ctypes.c_double), ("cdrho", ctypes.c_double),
                ("cimpd", ctypes.c_double), ("tend", ctypes.c_double),
                ("sedov_energy", ctypes.c_double), ("rho0", ctypes.POINTER(ctypes.c_double)),
                ("nrz", ctypes.c_int)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        _lib.o_delt.restype = ctypes.c_double
        _lib.o_run.restype = ctypes.c_int
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


class Oracle:
    """Holds a mesh and a configuration; methods mirror the reference routines."""

    def __init__(self, mesh, cfg, rho0=None):
        """rho0: optional per-cell initial-density factors (ncell,)."""
        self.mesh, self.cfg = mesh, cfg
        self._rho0 = None if rho0 is None else np.ascontiguousarray(rho0, dtype=np.float64).reshape(-1)
        self._keep = [np.ascontiguousarray(a, dtype=np.int32) for a in
                      (mesh.iptri, mesh.ipqua, mesh.bface, mesh.esuv1, mesh.esuv2, mesh.esqua)]
        k = self._keep
        self.om = _OMesh(mesh.ntria, mesh.nquad, mesh.npoin, mesh.nbfac,
                         _p(k[0], _ip), _p(k[1], _ip), _p(k[2], _ip), _p(k[3], _ip), _p(k[4], _ip),
                         _p(k[5], _ip), int(getattr(mesh, "nvqua", 9)))
        sc = (ctypes.c_int * 4)(*(list(cfg.sedov_cells) + [0, 0, 0, 0])[:4])
        self.oc = _OCfg(cfg.npoly, cfg.ndegr, cfg.mdegr, cfg.nq, cfg.nstag, cfg.ndt, cfg.ncase,
                        cfg.nlimi, 1, cfg.ngausd, cfg.ngausd_geo, len(cfg.sedov_cells), sc,
                        cfg.gamlg, cfg.cfl, cfg.cdrho, cfg.cimpd, cfg.tend, cfg.sedov_energy,
                        _p(self._rho0, _dp), int(getattr(cfg, "nrz", 0)))

    # arrays are returned in C order with the Fortran memory layout:
    #   unkno (nsize, nq, ndegr), geoel (nsize, 24), amatr (ncell, nmatr), coord (npoin, 2)
    def init(self):
        m, c = self.mesh, self.cfg
        geoel = np.zeros((m.nsize, 24))
        amatr = np.zeros((m.ncell, c.nmatr))
        unkno = np.zeros((m.nsize, c.nq, c.ndegr))
        coord = np.ascontiguousarray(m.coord)
        lib().o_init(ctypes.byref(self.om), ctypes.byref(self.oc), _p(coord, _dp), _p(geoel, _dp),
                     _p(amatr, _dp), _p(unkno, _dp))
        return geoel, amatr, unkno

    def cellvol(self, geoel, coord):
        lib().o_cellvol(ctypes.byref(self.om), ctypes.byref(self.oc), _p(geoel, _dp), _p(coord, _dp))

    def rhs(self, ustar, unkno, geoel, coord, coold, amatr, itime=1):
        m, c = self.mesh, self.cfg
        rhsel = np.zeros((m.ncell, c.nq, c.ndegr))
        flags = np.zeros(m.ncell, dtype=np.int32)
        lib().o_rhs(ctypes.byref(self.om), ctypes.byref(self.oc), _p(ustar, _dp), _p(unkno, _dp),
                    _p(rhsel, _dp), _p(geoel, _dp), _p(coord, _dp), _p(coold, _dp), _p(amatr, _dp),
                    ctypes.c_int(itime), _p(flags, _ip))
        return rhsel, flags

    def weno(self, unkno, geoel, coord, coold, flags):
        f = np.ascontiguousarray(flags, dtype=np.int32)
        lib().o_weno(ctypes.byref(self.om), ctypes.byref(self.oc), _p(unkno, _dp), _p(geoel, _dp),
                     _p(coord, _dp), _p(coold, _dp), _p(f, _ip))

    def error_norms(self, unkno, geoel, coord):
        """geterror_lag_curvhybrid's L2 errors (3,) on the quads."""
        e = np.zeros(3)
        lib().o_error(ctypes.byref(self.om), ctypes.byref(self.oc), _p(np.ascontiguousarray(unkno), _dp),
                      _p(np.ascontiguousarray(geoel), _dp), _p(np.ascontiguousarray(coord), _dp), _p(e, _dp))
        return e

    def rhs_p1(self, ustar, unkno, geoel, coord):
        """The linear P1 branch of getrhsdg_lag_mcnew; unkno is limited and
        ustar updated in place.  Returns (rhsel, aflim (ncell, 5), afvec (ncell, 4))."""
        m, c = self.mesh, self.cfg
        rhsel = np.zeros((m.ncell, c.nq, c.ndegr))
        aflim = np.zeros((m.ncell, 5))
        afvec = np.zeros((m.ncell, 4))
        lib().o1_rhs(ctypes.byref(self.om), ctypes.byref(self.oc), _p(ustar, _dp), _p(unkno, _dp),
                     _p(rhsel, _dp), _p(geoel, _dp), _p(coord, _dp), _p(aflim, _dp), _p(afvec, _dp))
        return rhsel, aflim, afvec

    @staticmethod
    def status() -> int:
        return int(lib().o_status())

    @staticmethod
    def counts():
        """(Persson-marked quads, WENO-replaced quads) summed over every stage
        since the previous call; resets both."""
        a, b = ctypes.c_longlong(0), ctypes.c_longlong(0)
        lib().o_counts(ctypes.byref(a), ctypes.byref(b))
        return int(a.value), int(b.value)

    def delt(self, unkno, geoel, coord, dvdt, itime, dtfix):
        return lib().o_delt(ctypes.byref(self.om), ctypes.byref(self.oc), _p(unkno, _dp), _p(geoel, _dp),
                            _p(coord, _dp), _p(dvdt, _dp), ctypes.c_int(itime), ctypes.c_double(dtfix))

    def run(self, unkno, coord, coold, geoel, amatr, ustar, itime0, nsteps, dtfix, tacru):
        """Driver loop; arrays updated in place. Returns (steps_done, dtfix, tacru)."""
        dt = ctypes.c_double(dtfix)
        ta = ctypes.c_double(tacru)
        n = lib().o_run(ctypes.byref(self.om), ctypes.byref(self.oc), _p(unkno, _dp), _p(coord, _dp),
                        _p(coold, _dp), _p(geoel, _dp), _p(amatr, _dp), _p(ustar, _dp),
                        ctypes.c_int(itime0), ctypes.c_int(nsteps), ctypes.byref(dt), ctypes.byref(ta))
        return n, dt.value, ta.value
