"""The block-inverse solve kernels agree.

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


@pytest.mark.parametrize("name", list(CASES))
def test_tensor_core_solve_matches_grouped_solve(name):
    """The grouped solve with its block products on the FP64 tensor cores
    (mma.sync m8n8k4) applies the same operators; only the rounding of each
    product differs (1e-12 of the field in FP64 after 5 steps, 1e-5 in mixed
    precision, where the FP32 storage rounds the difference up)."""
    import iwrepo_b200 as iw
    cfg = cf.Config(dt=1e-3, **CASES[name]).validate()
    runs = []
    for variant in (1, 2):
        s = iw.Solver(cfg)
        s.set_launch("solve", variant)
        s.init_mode1(0.05, 1e-3, 17)
        s.step(5)
        runs.append([s.state(lev) for lev in range(5)])
        s.close()
    tol = 1e-12 if cfg.precision == cf.IW_PREC_FP64 else 1e-5
    for a, b in zip(*runs):
        for q in range(4):
            n = np.linalg.norm(a[q])
            assert np.linalg.norm(a[q] - b[q]) <= tol * (n if n > 0 else 1.0), (name, q)


@pytest.mark.parametrize("name", list(CASES))
def test_two_row_solve_equals_grouped_solve(name):
    """The grouped solve with two rows per thread (variant 3: u/v, w and rho;
    the pressure keeps variant 1) runs every sum of the one-row grouped kernel
    in the same order: identical states after 5 steps.  At 512 rows (16
    subdomains of 32) the row pairs do not fit one CTA and the one-row kernel
    runs, which the test covers too."""
    import iwrepo_b200 as iw
    cfg = cf.Config(dt=1e-3, **CASES[name]).validate()
    runs = []
    for variant in (1, 3):
        s = iw.Solver(cfg)
        s.set_launch("solve", variant)
        s.init_mode1(0.05, 1e-3, 17)
        s.step(5)
        runs.append([s.state(lev) for lev in range(5)])
        s.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b), name


def test_per_role_solve_choices():
    """iw_set_launch / iw_get_launch per solve role; a role given variant 3
    matches the run with every role on the one-row grouped kernel."""
    import iwrepo_b200 as iw
    cfg = cf.Config(dt=1e-3, **CASES["c3-vertical-mixed"]).validate()
    a, b = iw.Solver(cfg), iw.Solver(cfg)
    a.set_launch("solve", 1)
    b.set_launch("solve", 1)
    for role in ("uv", "w", "rho"):
        b.set_launch("solve_" + role, 3)
        assert b.get_launch("solve_" + role) == 3
    assert b.get_launch("solve_pressure") == -1
    for s in (a, b):
        s.init_mode1(0.05, 1e-3, 5)
        s.step(4)
    assert np.array_equal(a.state(0), b.state(0))
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [cf.IW_PREC_FP64, cf.IW_PREC_MIXED])
@pytest.mark.parametrize("nzloc", [17, 25, 33])
def test_stage_e_variants_agree(precision, nzloc):
    """Stage E as a tiled kernel (0), a register-column kernel (1), the
    tiled kernel with its input tiles staged by bulk asynchronous copies (2),
    or that kernel with its operators in the constant bank (3).
    They run the same sums in the same order and differ in how the compiler
    contracts the products (1e-11 of the field in FP64, 1e-5 in mixed
    precision after 4 steps)."""
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=16, ny=16, nzloc=nzloc, nsubd=3, dt=1e-3, precision=precision).validate()
    runs = {}
    for variant in (0, 1, 2, 3):
        s = iw.Solver(cfg)
        s.set_launch("stage_e", variant)
        s.init_mode1(0.05, 1e-3, 23)
        s.step(4)
        runs[variant] = [s.state(lev) for lev in range(5)]
        s.close()
    tol = 1e-11 if precision == cf.IW_PREC_FP64 else 1e-5
    for a, b in zip(runs[2], runs[3]):  # the same sums from the same operator values
        assert np.array_equal(a, b)
    for v in runs:
        for a, b in zip(runs[0], runs[v]):
            for q in range(4):
                n = np.linalg.norm(a[q])
                assert np.linalg.norm(a[q] - b[q]) <= tol * (n if n > 0 else 1.0), (v, q)


@pytest.mark.parametrize("precision", [cf.IW_PREC_FP64, cf.IW_PREC_MIXED])
def test_stage_a_variants_give_the_same_bits(precision):
    """Stage A as a tiled kernel (0) or a register-column kernel (1): the same
    sums in the same order with every rounding written out, so the same bits."""
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=16, ny=16, nzloc=17, nsubd=3, dt=1e-3, precision=precision).validate()
    runs = []
    for variant in (0, 1):
        s = iw.Solver(cfg)
        s.set_launch("stage_a", variant)
        s.init_mode1(0.05, 1e-3, 29)
        s.step(4)
        runs.append([s.state(lev) for lev in range(5)])
        s.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_autotune_reports_the_solve_variant():
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=32, ny=32, nzloc=17, nsubd=4, dt=1e-3, precision=cf.IW_PREC_MIXED).validate()
    s = iw.Solver(cfg)
    s.init_mode1(0.05, 1e-4, 3)
    ch = s.autotune()
    kinds = ("system-grouped", "system-grouped-tensor-core", "per-task", "system-grouped-two-rows")
    assert ch["solve"] in kinds
    assert set(ch["solve_roles"]) == {"uv", "w", "rho", "pressure"}
    assert all(v in kinds for v in ch["solve_roles"].values())
    assert ch["solve_roles"]["pressure"] != "system-grouped-two-rows"
    s.step(2)
    s.close()


@pytest.mark.parametrize("precision", [cf.IW_PREC_FP64, cf.IW_PREC_MIXED])
@pytest.mark.parametrize("nx", [32, 48, 256])
def test_x_row_threads_give_the_same_bits(precision, nx):
    """k_xrow_nl with 256 or 128 threads per CTA: every loop strides by the
    block size and every element sees the same arithmetic, so the same bits
    (power-of-two lengths with compile-time plans and a mixed-radix length)."""
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=nx, ny=16, nzloc=9, nsubd=3, dt=1e-3, precision=precision).validate()
    runs = []
    for xt in (256, 128):
        s = iw.Solver(cfg)
        s.set_launch("x_row_threads", xt)
        assert s.get_launch("x_row_threads") == xt
        s.init_mode1(0.05, 1e-3, 41)
        s.step(3)
        runs.append(s.state(0))
        s.close()
    assert np.array_equal(runs[0], runs[1])
