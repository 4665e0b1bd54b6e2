"""The two block-inverse solve kernels give the same bits.

k_solve_sys (one CTA per group of columns that share a system, tables staged
in shared memory by bulk copies) and k_solve_cta (one CTA per task of <= 4
right-hand sides) apply the same inverse blocks, interface system and
projection with every sum in the same order.  Steps with either kernel must
leave identical states, for every solve role (pressure with the residual
sweep prefix, u/v with the mean-u damping, w, rho), both boundary variants,
both precisions, subdomains of equal and unequal heights (1 to 12 distinct
blocks), and the largest row count the grouped kernel takes (512).
"""
import numpy as np
import pytest

from iwrepo_b200 import config as cf

pytestmark = pytest.mark.gpu

CASES = {
    "equal-fp64-noslip": dict(nx=32, ny=32, nzloc=9, nsubd=3, precision=cf.IW_PREC_FP64),
    "equal-mixed-noslip": dict(nx=32, ny=32, nzloc=9, nsubd=3, precision=cf.IW_PREC_MIXED),
    "unequal-fp64-freeslip": dict(nx=16, ny=16, nzloc=13, nsubd=4, precision=cf.IW_PREC_FP64,
                                  bc_variant=cf.IW_BC_FREESLIP, z0=[0.0, 0.1, 0.3, 0.6], zh=[0.1, 0.2, 0.3, 0.4]),
    "c3-vertical-mixed": dict(nx=16, ny=16, nzloc=33, nsubd=12, precision=cf.IW_PREC_MIXED),
    "one-subdomain": dict(nx=16, ny=8, nzloc=17, nsubd=1, precision=cf.IW_PREC_FP64),
    "512-rows-fp64": dict(nx=8, ny=8, nzloc=32, nsubd=16, precision=cf.IW_PREC_FP64),
}


@pytest.mark.parametrize("name", list(CASES))
def test_grouped_solve_equals_per_task_solve(name):
    import iwrepo_b200 as iw
    cfg = cf.Config(dt=1e-3, **CASES[name]).validate()
    runs = []
    for variant in (0, 1):
        s = iw.Solver(cfg)
        s.set_launch("solve", variant)
        s.init_mode1(0.05, 1e-3, 17)
        s.step(5)
        runs.append([s.state(lev) for lev in range(5)])
        s.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b), name


def test_autotune_reports_the_solve_variant():
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=32, ny=32, nzloc=17, nsubd=4, dt=1e-3, precision=cf.IW_PREC_MIXED).validate()
    s = iw.Solver(cfg)
    s.init_mode1(0.05, 1e-4, 3)
    ch = s.autotune()
    assert ch["solve"] in ("system-grouped", "per-task")
    s.step(2)
    s.close()
