"""lag2d_delt_noalloc (the allocation-free getdelt_lag) against lag2d_step.

Collected last (file name) so it also runs after the other GPU tests in the
same process.  For two time steps in a row, the state at the start of the
step is taken from one handle; lag2d_rhs on a second handle gives the
limited stage state and dvdt = rhsel(1,1,:) exactly as the step computes
them; lag2d_delt_noalloc on caller-owned device copies of those arrays must
give the dtfix lag2d_step returns (bit for bit in the no-FMA build, within
1e-14 relative in the FMA build, where the compiler may contract the two
kernels' arithmetic differently).  Curved 9-node quads (ncurv = 1) and the
straight 4-node quads of the linear P1 path (ncurv = 0) are both covered.
"""
import ctypes

import numpy as np
import pytest

from lag2d_b200 import workload
from lag2d_b200 import api as _api
from lag2d_b200.api import Lag2DSolver

pytestmark = pytest.mark.gpu

MAX_QUADS = 4194304   # LAG2D_DELT_NOALLOC_MAX_QUADS


def _noalloc(lib):
    f = lib.lag2d_delt_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 8 + [ctypes.c_void_p] * 5 + [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                                ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    return f


def _layout(m):
    """(nvqua, ncurv) of the mesh: 9-node curved quads or 4-node straight ones."""
    nvqua = m.ipqua.shape[1]
    return nvqua, (0 if nvqua == 4 else 1)


def _call(f, m, c, dev, itime, dtfix_d):
    nvqua, ncurv = _layout(m)
    ngeel = dev["geoel"].shape[1]
    return f(m.ntria, m.nquad, m.npoin, nvqua, ncurv, c.ndegr, c.nq, ngeel, dev["ipqua"].data_ptr(),
             dev["unkno"].data_ptr(),
             dev["geoel"].data_ptr(), dev["coord"].data_ptr(), dev["dvdt"].data_ptr(), itime, c.ndens,
             c.gamlg, c.cfl, dtfix_d.data_ptr(), None)


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("name", ["tgv16", "sedov16", "sod_jitter40"])
def test_delt_noalloc_matches_step(name, exact):
    torch = pytest.importorskip("torch")
    m, c = workload(name)
    stepper = Lag2DSolver(m, c, exact=exact)
    f = _noalloc(stepper.lib)
    stepper.init_fields()
    ipq = torch.from_numpy(np.ascontiguousarray(m.ipqua, dtype=np.int32)).cuda()
    dtfix, tacru = c.dtfix, 0.0
    for itime in (1, 2):
        # a second handle brought to the same state (the step is deterministic)
        probe = Lag2DSolver(m, c, exact=exact)
        probe.init_fields()
        pdt, pta = c.dtfix, 0.0
        for k in range(1, itime):
            pdt, pta = probe.step(itime=k, dtfix=pdt, tacru=pta)
        geoel = probe.get_state()[3]            # geoel(3, :) = volume at the step start
        rhsel, _ = probe.rhs(itime=itime)       # stage-1 RHS, state limited in place
        ulim, coord = probe.get_state()[:2]
        probe.close()
        dev = {"ipqua": ipq,
               "unkno": torch.from_numpy(ulim).cuda(),
               "geoel": torch.from_numpy(geoel).cuda(),
               "coord": torch.from_numpy(coord).cuda(),
               "dvdt": torch.from_numpy(np.ascontiguousarray(rhsel[:, 0, 0])).cuda()}
        dt_d = torch.tensor([dtfix], dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = _call(f, m, c, dev, itime, dt_d)
        assert rc == 0, stepper.lib.lag2d_last_error()
        torch.cuda.synchronize()
        got = float(dt_d.cpu()[0])
        dtfix, tacru = stepper.step(itime=itime, dtfix=dtfix, tacru=tacru)
        if exact:
            assert got == dtfix, (itime, got, dtfix)
        else:
            assert abs(got - dtfix) <= 1e-14 * dtfix, (itime, got, dtfix)
    stepper.close()


def test_delt_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    lib = _api.load(False)
    f = _noalloc(lib)
    d = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = f(0, MAX_QUADS + 1, 9, 9, 1, 6, 4, 24, d.data_ptr(), d.data_ptr(), d.data_ptr(), d.data_ptr(), d.data_ptr(),
           1, 1, 1.4, 0.1, d.data_ptr(), None)
    assert rc == 1
    assert b"LAG2D_DELT_NOALLOC_MAX_QUADS" in lib.lag2d_last_error()


def test_delt_noalloc_empty_mesh():
    """nquad = 0: both minima stay at 1e10 (Getrhslag.f90:20637-20638)."""
    torch = pytest.importorskip("torch")
    lib = _api.load(False)
    f = _noalloc(lib)
    d = torch.full((1,), 5.0, dtype=torch.float64, device="cuda")
    rc = f(0, 0, 0, 9, 1, 6, 4, 24, None, None, None, None, None, 2, 1, 1.4, 0.1, d.data_ptr(), None)
    assert rc == 0, lib.lag2d_last_error()
    torch.cuda.synchronize()
    assert float(d.cpu()[0]) == min(0.1 * 1e10, 0.1 * 1e10, 1.01 * 5.0)


@pytest.mark.parametrize("nvqua,ncurv", [(4, 1), (8, -1), (3, 0)])
def test_delt_noalloc_rejects_layout(nvqua, ncurv):
    """ipqua with fewer entries per quad than the edge rule of ncurv reads
    (4 for straight edges, 8 for curved ones), or a negative ncurv, is
    rejected before any device work."""
    torch = pytest.importorskip("torch")
    lib = _api.load(False)
    f = _noalloc(lib)
    d = torch.full((64,), 1.0, dtype=torch.float64, device="cuda")
    rc = f(0, 1, 9, nvqua, ncurv, 3, 4, 24, d.data_ptr(), d.data_ptr(), d.data_ptr(), d.data_ptr(), d.data_ptr(),
           1, 1, 1.4, 0.1, d.data_ptr(), None)
    assert rc == 1
    assert b"ncurv" in lib.lag2d_last_error()


@pytest.mark.parametrize("bad_id", [0, "npoin+1"])
def test_delt_noalloc_bad_node_id_gives_nan(bad_id):
    """A node id outside 1..npoin in ipqua is not dereferenced: the call
    succeeds and dtfix comes back NaN (followed by a call on the intact mesh,
    so the scratch left by the first call does not leak into the second)."""
    torch = pytest.importorskip("torch")
    m, c = workload("tgv16")
    s = Lag2DSolver(m, c)
    f = _noalloc(s.lib)
    s.init_fields()
    geoel = s.get_state()[3]
    rhsel, _ = s.rhs(itime=1)
    ulim, coord = s.get_state()[:2]
    s.close()
    ipq = np.ascontiguousarray(m.ipqua, dtype=np.int32).copy()
    ipq[m.nquad // 2, 4] = 0 if bad_id == 0 else m.npoin + 1
    good = {"ipqua": torch.from_numpy(np.ascontiguousarray(m.ipqua, dtype=np.int32)).cuda(),
            "unkno": torch.from_numpy(ulim).cuda(), "geoel": torch.from_numpy(geoel).cuda(),
            "coord": torch.from_numpy(coord).cuda(),
            "dvdt": torch.from_numpy(np.ascontiguousarray(rhsel[:, 0, 0])).cuda()}
    bad = dict(good, ipqua=torch.from_numpy(ipq).cuda())
    for dev, expect_nan in ((bad, True), (good, False)):
        dt_d = torch.tensor([c.dtfix], dtype=torch.float64, device="cuda")
        rc = _call(f, m, c, dev, 1, dt_d)
        assert rc == 0, s.lib.lag2d_last_error()
        torch.cuda.synchronize()
        got = float(dt_d.cpu()[0])
        assert np.isnan(got) == expect_nan, got
