"""CPU checks of the C-ABI library: it loads, exports every entry point that
include/lag2d.h declares, and validates arguments before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from lag2d_b200 import api, workload

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "lag2d.h")).read()
    return sorted(set(re.findall(r"\b(lag2d_[a-z0-9_]+)\s*\(", txt)))


@pytest.mark.parametrize("exact", [False, True])
def test_library_exports_header_symbols(exact):
    lib = ctypes.CDLL(api.library_path(exact))
    names = _declared()
    assert "lag2d_step" in names and "lag2d_create" in names
    for n in names:
        assert hasattr(lib, n), n
    assert set(api.EXPORTS) <= set(names)


def test_create_validates_arguments_without_device():
    lib = api.load()
    h = ctypes.c_void_p()
    rc = lib.lag2d_create(None, None, ctypes.byref(h))
    assert rc == 1 and b"null" in lib.lag2d_last_error()
    m, c = workload("tgv16")
    s = object.__new__(api.Lag2DSolver)
    # a mesh with an out-of-range node id is rejected before any CUDA call
    bad = m.ipqua.copy()
    bad[0, 0] = m.npoin + 5
    k = [np.ascontiguousarray(a, dtype=np.int32) for a in (m.iptri, bad, m.bface, m.esuv1, m.esuv2, m.esqua)]
    coold = np.ascontiguousarray(m.coord)
    mm = api._Mesh(m.ntria, m.nquad, m.npoin, m.nbfac, *[api._p(a, api._ip) for a in k], api._p(coold, api._dp))
    cc = api._Cfg(c.npoly, c.ndegr, c.mdegr, c.nq, c.nstag, c.ndt, c.ncase, c.nlimi, c.ndens, c.ngausd,
                  c.ngausd_geo, 0, 0, 0, (ctypes.c_int * 4)(), c.gamlg, c.cfl, c.cdrho, c.cimpd, c.tend,
                  c.sedov_energy)
    assert lib.lag2d_create(ctypes.byref(mm), ctypes.byref(cc), ctypes.byref(h)) == 1
    # invalid and unsupported configurations are reported as such
    k[1] = np.ascontiguousarray(m.ipqua, dtype=np.int32)
    mm.ipqua = api._p(k[1], api._ip)
    cc.precision = 2
    assert lib.lag2d_create(ctypes.byref(mm), ctypes.byref(cc), ctypes.byref(h)) == 1
    cc.precision, cc.order_exact = 1, 1      # the reference-order kernels are FP64 only
    assert lib.lag2d_create(ctypes.byref(mm), ctypes.byref(cc), ctypes.byref(h)) == 1
    cc.precision, cc.order_exact = 0, 0
    cc.npoly, cc.ndegr, cc.mdegr = 1, 3, 6   # the P1 path: mdegr must be <= 3
    assert lib.lag2d_create(ctypes.byref(mm), ctypes.byref(cc), ctypes.byref(h)) == 1
    cc.mdegr = 3                             # the P1 path has no Taylor-Green source
    assert lib.lag2d_create(ctypes.byref(mm), ctypes.byref(cc), ctypes.byref(h)) == 3
    cc.npoly, cc.ndegr, cc.mdegr = c.npoly, c.ndegr, c.mdegr
    cc.nstag = 4
    assert lib.lag2d_create(ctypes.byref(mm), ctypes.byref(cc), ctypes.byref(h)) == 1
    del s


def test_rz_configurations_rejected_without_device():
    """RZ is built on the linear P1 path: P2 with nrz = 1 or 2 and the RZ
    Sedov case (a hard-coded dt schedule) in either RZ form return
    LAG2D_EUNSUP (3) before any device work; nrz = 3 is LAG2D_EINVAL (1)."""
    import dataclasses
    lib = api.load()
    cases = (("tgv16", {"nrz": 1}, 3), ("tgv16", {"nrz": 2}, 3), ("noh_rz8", {"ncase": 7}, 3),
             ("noh_rz8", {"nrz": 2, "ncase": 7}, 3), ("noh_rz8", {"nrz": 3}, 1))
    for name, change, rc in cases:
        m, c = workload(name)
        c = dataclasses.replace(c, **change)
        k = [np.ascontiguousarray(a, dtype=np.int32) for a in (m.iptri, m.ipqua, m.bface, m.esuv1, m.esuv2, m.esqua)]
        coold = np.ascontiguousarray(m.coord)
        mm = api._Mesh(m.ntria, m.nquad, m.npoin, m.nbfac, *[api._p(a, api._ip) for a in k],
                       api._p(coold, api._dp))
        cc = api._Cfg(c.npoly, c.ndegr, c.mdegr, c.nq, c.nstag, c.ndt, c.ncase, c.nlimi, c.ndens, c.ngausd,
                      c.ngausd_geo, 0, 0, 0, (ctypes.c_int * 4)(), c.gamlg, c.cfl, c.cdrho, c.cimpd, c.tend,
                      c.sedov_energy, c.nrz)
        h = ctypes.c_void_p()
        assert lib.lag2d_create(ctypes.byref(mm), ctypes.byref(cc), ctypes.byref(h)) == rc, (name, change)
        assert b"RZ" in lib.lag2d_last_error() or b"nrz" in lib.lag2d_last_error()


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(api, "_LIBDIR", str(tmp_path))
    monkeypatch.setattr(api, "_libs", {})
    with pytest.raises(FileNotFoundError):
        api.load()


def test_entry_points_reject_null_handles_without_device():
    """Every handle entry point returns LAG2D_EINVAL for a null handle before
    any CUDA call (the adjoint and density-hook entries included)."""
    lib = api.load()
    d = ctypes.c_double(0.0)
    buf = np.zeros(8)
    p = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert lib.lag2d_step(None, 1, ctypes.byref(d), ctypes.byref(d)) == 1
    assert lib.lag2d_set_rho0(None, p) == 1
    assert lib.lag2d_error_norms(None, p) == 1
    assert lib.lag2d_cell_output(None, p, p) == 1
    assert lib.lag2d_adjoint(None, 1, 2, 1, ctypes.byref(d), ctypes.byref(d), ctypes.byref(d),
                             None, None, None, None) == 1
    assert lib.lag2d_adjoint_step(None, 1, ctypes.byref(d), ctypes.byref(d), None, None, None,
                                  None, None, None) == 1
    assert b"null" in lib.lag2d_last_error()
