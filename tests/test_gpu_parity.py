"""GPU parity of the B200 library against the CPU oracle (through the C ABI).

Tolerances:
* drop-in routines: horfft_/dpdz_ 1e-14 relative L2; penalty_main_ and
  bandlu_solve_ bit-identical (same LAPACK arithmetic, no FMA);
* full steps, FP64: <= 1e-10 relative L2 per field after 100 steps of C0
  (64^2 x (4x17)), KE and dissipation time series to 1e-10;
* the oracle can apply the Fourier filter as a plain scale instead of the
  reference's magnitude/phase form (identical in exact arithmetic); against
  that form the GPU agrees to 1e-12 after 20 steps in every field;
* mixed precision: <= 1e-5 relative L2 vs the FP64 GPU path after 100 steps.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


@pytest.fixture(scope="module")
def small():
    from iwrepo_b200 import config as cf
    return cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=1e-3).validate()


def test_library_loaded_and_cuda_path(small):
    import iwrepo_b200 as iw
    s = iw.Solver(small)
    assert s.device_bytes() > 0
    assert s.field_ptr(0) != 0


def test_horfft_dpdz(small):
    import iwrepo_b200 as iw
    from oracle import Oracle
    o, s = Oracle(small), iw.Solver(small)
    rng = np.random.default_rng(0)
    ph = np.zeros((small.nz, small.ny, small.nxpp))
    ph[:, :, :small.nx] = rng.standard_normal((small.nz, small.ny, small.nx))
    assert rel(s.horfft(ph, -1), o.horfft(ph.copy(), -1)) < 1e-14
    sp = o.horfft(ph.copy(), -1)
    assert rel(s.horfft(sp, 1), o.horfft(sp.copy(), 1)) < 1e-14
    assert rel(s.dpdz(sp), o.dpdz(sp)) < 1e-14
    assert rel(s.filter_3dlegenfourier(sp), o.filter3d(sp)) < 1e-13
    assert rel(s.filter_3dlegenfourier(sp, 0, 1), o.filter3d(sp, 0, 1)) < 1e-14


@pytest.mark.parametrize("eps,bot,top", [(1e-2, 0, 0), (0.7, 1, 1), (1e-6, 0, 1), (2e-5, 1, 1), (1.0, 1, 1)])
def test_penalty_main_bit_identical(small, eps, bot, top):
    import iwrepo_b200 as iw
    from oracle import Oracle
    o, s = Oracle(small), iw.Solver(small)
    rng = np.random.default_rng(int(eps * 1e6) + bot)
    r1, r2 = rng.standard_normal(small.nz), rng.standard_normal(small.nz)
    bcs = (0.3, -0.2, 0.1, 0.05) if bot == 1 else (0.0, 0.0, 0.0, 0.0)
    s.penalty_setup(eps)
    o.penalty_setup(eps)
    fr, fi, rr, _ = s.penalty_main(eps, bot, top, bcs, r1, r2)
    gr, gi, qr, _ = o.penalty_main(eps, bot, top, bcs, r1, r2)
    assert np.array_equal(fr, gr) and np.array_equal(fi, gi)
    assert np.array_equal(rr, qr)  # rhs scaled by -eps in place


def test_bandlu_solve_bit_identical(small):
    import iwrepo_b200 as iw
    from oracle import Oracle
    o, s = Oracle(small), iw.Solver(small)
    A = o.penalty_matrix(3e-3, 0, 1)
    rng = np.random.default_rng(3)
    x1, x2 = rng.standard_normal(small.nz), rng.standard_normal(small.nz)
    a, b = s.bandlu_solve(A, x1, x2)
    assert np.linalg.norm(A @ a - x1) / np.linalg.norm(x1) < 1e-12
    o.penalty_setup(3e-3)
    fr, fi, _, _ = o.penalty_main(3e-3, 0, 1, (0, 0, 0, 0), -x1 / 3e-3, -x2 / 3e-3)
    assert np.max(np.abs(A @ fr - x1)) < 1e-9
    import ctypes
    import oracle
    xr, xi = x1.copy(), x2.copy()
    pd = ctypes.POINTER(ctypes.c_double)
    oracle.lib().orc_bandlu_solve(o.h, np.ascontiguousarray(A.T).ctypes.data_as(pd), xr.ctypes.data_as(pd),
                                  xi.ctypes.data_as(pd))
    assert np.array_equal(a, xr) and np.array_equal(b, xi)


def test_interface_avg3d(small):
    import iwrepo_b200 as iw
    from oracle import Oracle
    o, s = Oracle(small), iw.Solver(small)
    rng = np.random.default_rng(5)
    ph = np.zeros((small.nz, small.ny, small.nxpp))
    ph[:, :, :small.nx] = rng.standard_normal((small.nz, small.ny, small.nx))
    sp = o.horfft(ph, -1)
    g1, ic1 = s.interface_avg3d(sp)
    g2, ic2 = o.interface_avg3d(sp)
    assert ic1 == ic2 and ic1 > 0
    assert rel(g1, g2) < 1e-14


def run_pair(cfg, steps, fourier_scale, seed=5, amp=0.05, noise=1e-4):
    import iwrepo_b200 as iw
    from oracle import Oracle
    o, s = Oracle(cfg, fourier_scale=fourier_scale), iw.Solver(cfg)
    o.init_mode1(amp, noise, seed)
    s.init_mode1(amp, noise, seed)
    o.step(steps)
    s.step(steps)
    return s, o


@pytest.mark.parametrize("solver", [0, 1])
def test_steps_3d_strict(small, solver):
    """solver 0: block inverses for the viscous systems; 1: banded LU for all."""
    s, o = run_pair(small.replace(solver=solver), 20, fourier_scale=True)
    a, b = s.state(), o.state()
    for q in range(4):
        assert rel(a[q], b[q]) < (1e-11 if q == 1 else 1e-12), q  # v is a small (noise-only) field
    for lev in (1, 2, 3, 4):  # histories
        a, b = s.state(lev), o.state(lev)
        for q in range(4):
            assert rel(a[q], b[q]) < 1e-11, (lev, q)


def test_diag_maxcalc_and_bottom_rms_match_oracle(small):
    """iw_diag: CFL (various.f:665-987, incl. the merged-interface dz), extrema
    and the rms of w below 0.2 zlen, against the oracle on the same state."""
    s, o = run_pair(small, 5, fourier_scale=True)
    d = s.diag()
    o.maxcalc()
    m = o.last_maxcalc()
    assert np.allclose(d["cfl"], m["cfl"], rtol=1e-10, atol=1e-300)
    mm = np.array(d["minmax"])
    keep = [0, 2, 3, 4, 5, 6, 7]  # the reference's running umax adds an offset (umax) and is not reproduced
    assert np.allclose(mm[keep], m["minmax"][keep], rtol=1e-10, atol=1e-14)
    assert abs(d["wrms_bottom"] - o.diag()["wrms_bottom"]) <= 1e-10 * o.diag()["wrms_bottom"]
    assert abs(d["ke"] - o.diag()["ke"]) <= 1e-10 * o.diag()["ke"]


def test_steps_3d_faithful_filter(small):
    s, o = run_pair(small, 20, fourier_scale=False)
    a, b = s.state(), o.state()
    for q in range(4):
        assert rel(a[q], b[q]) < 1e-10, q


@pytest.mark.parametrize("variant", [0, 1])
def test_steps_2d_and_variants(variant):
    from iwrepo_b200 import config as cf
    cfg = cf.Config(nx=32, ny=1, nzloc=9, nsubd=4, dt=1e-3, bc_variant=variant).validate()
    s, o = run_pair(cfg, 20, fourier_scale=False)
    a, b = s.state(), o.state()
    for q in range(4):
        assert rel(a[q], b[q]) < 1e-12, q


def test_forced_2d_shipped_config():
    """The shipped 2-D forced run (virtual paddle, 12 uneven subdomains)."""
    from iwrepo_b200 import config as cf
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = cf.shipped_2d(nx=64, bc_variant=cf.IW_BC_NOSLIP)
    o, s = Oracle(cfg, fourier_scale=True), iw.Solver(cfg)
    o.step(5)
    s.step(5)
    a, b = s.state(), o.state()
    for q in (0, 2, 3):
        assert rel(a[q], b[q]) < 1e-9, q


def test_c0_100_steps_parity_and_energy():
    """C0: 64^2 x (4x17), Re=1000, A=0.05, noise 1e-4, dt=1e-3, 100 steps."""
    import oracle
    from iwrepo_b200 import config as cf
    import iwrepo_b200 as iw
    oracle.set_threads(oracle.max_threads())
    cfg = cf.baseline("C0")
    o, s = oracle.Oracle(cfg), iw.Solver(cfg)
    o.init_mode1(0.05, 1e-4, 2024)
    s.init_mode1(0.05, 1e-4, 2024)
    for chunk in (10, 40, 50):
        o.step(chunk)
        s.step(chunk)
        do, ds = o.diag(), s.diag()
        assert abs(ds["ke"] - do["ke"]) <= 1e-10 * abs(do["ke"])
        assert abs(ds["eps"] - do["eps"]) <= 1e-10 * abs(do["eps"])
    a, b = s.state(), o.state()
    for q in range(4):
        assert rel(a[q], b[q]) <= 1e-10, q


def test_mixed_precision_vs_fp64():
    from iwrepo_b200 import config as cf
    import iwrepo_b200 as iw
    c64 = cf.baseline("C0")
    c32 = c64.replace(precision=cf.IW_PREC_MIXED)
    a_s, b_s = iw.Solver(c32), iw.Solver(c64)
    for s in (a_s, b_s):
        s.init_mode1(0.05, 1e-4, 99)
        s.step(100)
    a, b = a_s.state(), b_s.state()
    for q in (0, 2, 3):
        assert rel(a[q], b[q]) <= 1e-5, q
    # velocity vector as a whole
    assert rel(a[:3], b[:3]) <= 1e-5
    # v only holds the seeded noise (1e-4 of the wave): the FP32 rounding of the
    # wave shifts the advected noise pattern, and FP32-sized differences decide
    # the interface averaging at points at its threshold
    assert rel(a[1], b[1]) <= 1e-3


@pytest.mark.xfail(strict=False, reason="v, the noise-only field, misses the 1e-5 metric gate in mixed precision: "
                                        "the FP32-stored wave advects it with a phase error and FP32-sized "
                                        "differences flip interface-averaging decisions (see the precision notes)")
def test_mixed_precision_v_within_metric_gate():
    """The metric's gate (<= 1e-5 relative L2 in every field) applied to v:
    kept as an expected failure so that the miss stays visible."""
    from iwrepo_b200 import config as cf
    import iwrepo_b200 as iw
    c64 = cf.baseline("C0")
    c32 = c64.replace(precision=cf.IW_PREC_MIXED)
    a_s, b_s = iw.Solver(c32), iw.Solver(c64)
    for s in (a_s, b_s):
        s.init_mode1(0.05, 1e-4, 99)
        s.step(100)
    assert rel(a_s.state()[1], b_s.state()[1]) <= 1e-5


def test_deterministic():
    from iwrepo_b200 import config as cf
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=32, ny=32, nzloc=9, nsubd=3, dt=1e-3).validate()
    st = []
    for _ in range(2):
        s = iw.Solver(cfg)
        s.init_mode1(0.05, 1e-4, 3)
        s.step(7)
        st.append(s.state())
    assert np.array_equal(st[0], st[1])


def test_helm_batched_modes():
    """Isolated batched penalty solves (C1 shape reduced): FP64 factor+solve
    is the oracle's solve bit for bit; FP32 solve + one FP64 refinement has a
    small relative residual."""
    import torch
    from iwrepo_b200 import config as cf
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = cf.Config(nx=32, ny=32, nzloc=25, nsubd=8, dt=1e-3, xnu=1.0, xkappa=1.0).validate()
    s = iw.Solver(cfg)
    o = Oracle(cfg)
    kx = np.arange(cfg.nx // 2 + 1)
    ky = np.fft.fftfreq(cfg.ny, 1.0 / cfg.ny)
    lam = (kx[None, :] ** 2 + ky[:, None] ** 2).ravel() + 11.0 / (6 * cfg.dt)
    ncol = lam.size
    rng = np.random.default_rng(11)
    rhs = rng.standard_normal((ncol, cfg.nz, 2))
    dl = torch.tensor(lam, dtype=torch.float64, device="cuda")
    dr = torch.tensor(rhs, dtype=torch.float64, device="cuda")
    for mode in (0, 1):
        ds = torch.zeros_like(dr)
        iw.helm_solve_batched(s, dl.data_ptr(), ncol, 0, 1, dr.data_ptr(), ds.data_ptr(), mode)
        torch.cuda.synchronize()
        sol = ds.cpu().numpy()
        for c in (0, 1, 17, ncol - 1):
            A = o.penalty_matrix(1.0 / lam[c], 0, 1)
            res = np.linalg.norm(A @ sol[c, :, 0] - rhs[c, :, 0]) / np.linalg.norm(rhs[c, :, 0])
            assert res < (1e-11 if mode == 0 else 1e-7), (mode, c, res)
            if mode == 0:
                eps = 1.0 / lam[c]
                o.penalty_setup(eps)
                fr, fi, _, _ = o.penalty_main(eps, 0, 1, (0, 0, 0, 0), -rhs[c, :, 0] / eps, -rhs[c, :, 1] / eps)
                # the oracle's RHS went through (-b/eps)*(-eps): compare at rounding level
                assert np.max(np.abs(fr - sol[c, :, 0])) <= 1e-12 * np.max(np.abs(fr))


def test_config_errors_reported():
    import ctypes
    from iwrepo_b200 import config as cf
    import iwrepo_b200._lib as L
    cfg = cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=1e-3)
    d = cfg.c_dims()
    p = cfg.c_params()
    d.nx = 14 * 7  # radix 7
    h = ctypes.c_void_p()
    rc = L.lib().iw_init(ctypes.byref(d), ctypes.byref(p), 0, ctypes.byref(h))
    assert rc == 1 and b"nx" in L.lib().iw_last_error()
    d.nx = 16
    p.zh[0] = 0.1  # heights no longer add up to zlen
    rc = L.lib().iw_init(ctypes.byref(d), ctypes.byref(p), 0, ctypes.byref(h))
    assert rc == 1
