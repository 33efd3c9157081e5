"""lag2d_error_norms (geterror_lag_curvhybrid, Postprocess.f90:3587-4143) on
the device against the CPU restatement: the Taylor-Green L2 errors of rho,
|u| and p after a few steps, and the unsupported cases."""
import numpy as np
import pytest

from lag2d_b200 import workload
from lag2d_b200.api import Lag2DError, Lag2DSolver
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsteps", [0, 5])
def test_error_norms_match_oracle(nsteps):
    m, c = workload("tgv16")
    o = Oracle(m, c)
    geoel, amatr, unkno = o.init()
    coord = m.coord.copy()
    ustar = np.zeros_like(coord)
    if nsteps:
        o.run(unkno, coord, m.coord.copy(), geoel, amatr, ustar, 1, nsteps, c.dtfix, 0.0)
    e1 = o.error_norms(unkno, geoel, coord)
    s = Lag2DSolver(m, c)
    s.init_fields()
    if nsteps:
        s.run(nsteps)
    e2 = s.error_norms()
    # the device sums in a different order; the density error is rounding-level
    assert abs(e2[0] - e1[0]) < 1e-13
    assert np.all(np.abs(e2[1:] - e1[1:]) <= 1e-10 * e1[1:])


def test_error_norms_unsupported():
    m, c = workload("sedov16")
    s = Lag2DSolver(m, c)
    s.init_fields()
    with pytest.raises(Lag2DError) as e:
        s.error_norms()
    assert e.value.code == 3
