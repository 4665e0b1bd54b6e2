"""Failure detection inside the step, made on the host (no GPU fault).

* Non-finite state: a state uploaded with one NaN is found by the next step's
  stage A, which reads every value of the state; iw_sync reports
  IW_ERR_NONFINITE, later steps refuse to run, and a new state clears it.
* Zero pivot: bandlu_solve_ on a host-made matrix with an all-zero column
  records IW_ERR_PIVOT (iw_last_status), as SGBTF2's INFO would; the
  reference ignores INFO (band_lu.f:23-34).
* Deterministic diagnostics: iw_diag's KE and dissipation come from per-block
  sums added in a fixed order, so repeated calls give the same bits.
"""
import numpy as np
import pytest

from iwrepo_b200 import config as cf

pytestmark = pytest.mark.gpu

IW_ERR_NONFINITE, IW_ERR_PIVOT = 3, 4


@pytest.mark.parametrize("precision", [cf.IW_PREC_FP64, cf.IW_PREC_MIXED])
def test_nan_in_state_is_reported(precision):
    import iwrepo_b200 as iw
    from iwrepo_b200._lib import IwError
    cfg = cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=1e-3, precision=precision).validate()
    s = iw.Solver(cfg)
    s.init_mode1(0.05, 1e-4, 4)
    s.step(2)
    s.sync()  # a clean state: no error
    st = s.state(0)
    st[2, 5, 3, 6] = np.nan
    s.set_state(st, t=2 * cfg.dt, istep=2)
    s.sync()  # the upload alone is not checked
    s.step(1)  # stage A of this step reads the NaN
    with pytest.raises(IwError) as e:
        s.sync()
    assert e.value.code == IW_ERR_NONFINITE
    with pytest.raises(IwError) as e:  # the error is sticky: later steps refuse
        s.step(1)
    assert e.value.code == IW_ERR_NONFINITE
    s.init_mode1(0.05, 1e-4, 4)  # a new state clears it
    s.step(2)
    s.sync()
    s.close()


def test_zero_pivot_is_reported():
    import ctypes
    import iwrepo_b200 as iw
    from iwrepo_b200 import _lib
    cfg = cf.Config(nx=8, ny=2, nzloc=5, nsubd=2, dt=1e-3).validate()
    s = iw.Solver(cfg)
    n = cfg.nz
    A = np.eye(n) * 2.0 + np.diag(np.full(n - 1, 0.5), 1)
    A[:, 3] = 0.0  # column 4 is zero: SGBTF2 sets INFO = 4
    x1 = np.ones(n)
    s.bandlu_solve(A, x1, x1.copy())
    assert _lib.lib().iw_last_status() == IW_ERR_PIVOT
    assert b"pivot" in _lib.lib().iw_last_error()
    A[:, 3] = 0.0
    A[3, 3] = 1.0  # regular again
    s.bandlu_solve(A, x1, x1.copy())
    assert _lib.lib().iw_last_status() == 0
    s.close()


def test_diag_is_bitwise_repeatable():
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=64, ny=64, nzloc=17, nsubd=4, dt=1e-3, precision=cf.IW_PREC_MIXED).validate()
    s = iw.Solver(cfg)
    s.init_mode1(0.05, 1e-3, 8)
    s.step(3)
    d = [s.diag() for _ in range(4)]
    for x in d[1:]:
        assert x["ke"] == d[0]["ke"] and x["eps"] == d[0]["eps"]
    s.close()
