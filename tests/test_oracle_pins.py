"""Pin the CPU oracle to the reference's own numeric artefacts.

The reference has no test suite; its runs left text files that the oracle
must reproduce (tests/golden/reference_runs.json, made by make_golden.py):

* testout.dat (testhelm.f): penalty solve, 8 significant digits  -> exact pin
* z_grid.dat / x_grid.dat: GLL / uniform grids, 7 decimals        -> exact pin
* run log `output`: wave frequency of the 128x250 run, 15 digits  -> exact pin
* the recorded 400-step run (its log `output`, dtchange.dat and rows 641-1040
  of uveltest.dat): every input is printed in the log; the oracle reproduces
  its 16-digit probes u(32,1,10), u(32,1,50) and maxcalc's cflz at every step
  to 1e-9, with the paddle left out of the bottom point (IW_PADDLE_ABOVE_BOTTOM,
  the comment of solver.f:848-849).  With the paddle on every level, as the
  loop of solver.f:848 is written, they differ by 1e-4 from the first step.
* uveltest.dat / cfl.dat / minmaxtest.dat rows of a later 9-step run of the
  shipped 2-D forced configuration (calcuvwt_noslip.f).  The input.dat of that
  run is not recorded (it stopped after 9 of the 400 steps the shipped file
  asks for); the oracle follows it to 4-5 significant digits, the free-slip
  variant does not.
"""
import math

import numpy as np
import pytest

from iwrepo_b200 import config as cf
from oracle import Oracle, multistep


def runfolder_cfg(golden):
    sub = golden["subd_runfolder"]
    n = int(sub[0][0])
    z0 = [r[0] for r in sub[1:n + 1]]
    zh = [r[1] for r in sub[1:n + 1]]
    return cf.Config(nx=8, ny=1, nzloc=25, nsubd=n, dt=0.1, xlen=10.0, ylen=1.0, zlen=5.0,
                     z0=z0, zh=zh).validate()


def test_testhelm_testout(golden):
    """testhelm.f:59-99: eps=1e-2, rhs=-1, homogeneous Dirichlet both ends."""
    cfg = runfolder_cfg(golden)
    o = Oracle(cfg)
    eps = 1e-2
    o.penalty_setup(eps)
    nz = cfg.nz
    fr, fi, rr, _ = o.penalty_main(eps, 0, 0, (0.0, 0.0, 0.0, 0.0), -np.ones(nz), -np.ones(nz))
    ref = np.array(golden["testout"])
    z = o.tables()["z"]
    assert np.allclose(z, ref[:, 0], atol=6e-8, rtol=0)
    big = np.abs(ref[:, 1]) > 1e-6
    assert np.max(np.abs(fr[big] - ref[big, 1]) / np.abs(ref[big, 1])) < 1e-7
    assert np.max(np.abs(fr - ref[:, 1])) < 1e-10
    assert np.array_equal(fr, fi)
    # penalty_main scales the caller's RHS by -eps in place (penalty.f:188-191)
    assert np.allclose(rr, eps)
    # analytic solution of f - eps f'' = eps, f(0)=f(5)=0
    s = math.sqrt(eps)
    exact = eps * (1 - np.cosh((z - 2.5) / s) / math.cosh(2.5 / s))
    assert np.max(np.abs(fr - exact)) < 1e-9


def test_shipped_grids(golden):
    o = Oracle(cf.shipped_2d())
    z = o.tables()["z"]
    zr = np.array(golden["z_grid"])
    assert np.allclose(z, zr[:, 1], atol=6e-8, rtol=0)
    xr = np.array(golden["x_grid"])[:, 1]
    assert np.allclose(np.arange(256) * 20.0 / 256, xr, atol=6e-8)


def test_gll_tables_katp():
    cfg = cf.baseline("C0")
    t = Oracle(cfg).tables()
    zp, wg, d = t["zpts"], t["wg"], t["d"]
    assert abs(wg.sum() - 2.0) < 1e-14
    assert zp[0] == -1.0 and zp[-1] == 1.0
    # D is exact on polynomials of degree <= N
    for p in range(cfg.nzloc):
        assert np.allclose(d @ zp ** p, p * zp ** max(p - 1, 0) if p else 0 * zp, atol=1e-9)
    # GLL quadrature exact to degree 2N-1
    assert abs(wg @ zp ** 30 - 2.0 / 31) < 1e-13


@pytest.mark.parametrize("N", [9, 17, 25, 33])
def test_gll_tables_independent_derivation(N):
    """The GLL nodes, weights and differentiation matrix (setup.f:395-479,
    636-798) against a derivation that shares no code with the restatement:
    numpy's Legendre series, interior nodes = roots of P'_{N-1} (refined by
    Newton), w_j = 2 / (N (N-1) P_{N-1}(x_j)^2),
    D_kj = P_{N-1}(x_k) / (P_{N-1}(x_j) (x_k - x_j)), D_00 = -D_{N-1,N-1} =
    -N (N-1) / 4; D2 = D D, the exact second derivative on the GLL space."""
    from numpy.polynomial import legendre as leg
    t = Oracle(cf.Config(nx=16, ny=8, nzloc=N, nsubd=2, dt=1e-3).validate()).tables()
    c = np.zeros(N)
    c[-1] = 1.0
    r = np.sort(leg.legroots(leg.legder(c)))
    for _ in range(3):
        r -= leg.legval(r, leg.legder(c)) / leg.legval(r, leg.legder(c, 2))
    x = np.concatenate(([-1.0], r, [1.0]))
    p = leg.legval(x, c)
    w = 2.0 / (N * (N - 1) * p ** 2)
    d = np.zeros((N, N))
    for k in range(N):
        for j in range(N):
            if k != j:
                d[k, j] = p[k] / (p[j] * (x[k] - x[j]))
    d[0, 0], d[-1, -1] = -N * (N - 1) / 4.0, N * (N - 1) / 4.0
    assert np.abs(t["zpts"] - x).max() < 1e-15
    assert np.abs(t["wg"] - w).max() < 1e-15
    assert np.abs(t["d"] - d).max() < 5e-14 * np.abs(d).max()
    d2 = d @ d
    assert np.abs(t["d2"] - d2).max() < 1e-11 * np.abs(d2).max()


def test_wave_parameters_run_log():
    """output:53-67 of the 128x250 run: omega = 4.850712500726660E-002."""
    pi2 = 8 * math.atan(1.0)
    xk, xm = pi2 / 40.0, pi2 / (2 * 5.0)
    omega = (0.2 * xk) / math.sqrt(xk * xk + xm * xm)
    assert abs(omega - 4.850712500726660e-02) < 1e-16


def test_multistep_coefficients():
    dt = 0.37
    assert abs(multistep("abvar1", dt, dt, dt) - 23 / 12) < 1e-15
    assert abs(multistep("abvar2", dt, dt, dt) + 16 / 12) < 1e-15
    assert abs(multistep("abvar3", dt, dt, dt) - 5 / 12) < 1e-15
    assert abs(multistep("bdfvarv", dt, dt, dt) - 11 / 6) < 1e-15
    assert abs(multistep("bdfvar1", dt, dt, dt) - 3) < 1e-14
    assert abs(multistep("bdfvar2", dt, dt, dt) + 1.5) < 1e-14
    assert abs(multistep("bdfvar3", dt, dt, dt) - 1 / 3) < 1e-15


def test_horfft_semantics():
    """FFT991/CFFT99 conventions incl. the x-Nyquist column quirk."""
    cfg = cf.Config(nx=16, ny=8, nzloc=5, nsubd=2, dt=1e-3).validate()
    o = Oracle(cfg)
    rng = np.random.default_rng(1)
    phys = np.zeros((cfg.nz, cfg.ny, cfg.nxpp))
    phys[:, :, :cfg.nx] = rng.standard_normal((cfg.nz, cfg.ny, cfg.nx))
    spec = o.horfft(phys.copy(), -1)
    ref = np.fft.rfft2(phys[:, :, :cfg.nx], axes=(1, 2)) / (cfg.nx * cfg.ny)
    c = spec[:, :, 0::2] + 1j * spec[:, :, 1::2]
    assert np.allclose(c[:, :, :cfg.nx // 2], ref[:, :, :cfg.nx // 2], atol=1e-14)
    # Nyquist column: x-transformed only, then scaled by 1/ny
    nyq = np.fft.rfft(phys[:, :, :cfg.nx], axis=2)[:, :, cfg.nx // 2].real / cfg.nx / cfg.ny
    assert np.allclose(c[:, :, cfg.nx // 2].real, nyq, atol=1e-14)
    back = o.horfft(spec.copy(), 1)
    R = np.fft.rfft(phys[:, :, :cfg.nx], axis=2)
    R[:, :, cfg.nx // 2] /= cfg.ny  # a round trip scales the x-Nyquist column by 1/ny
    assert np.allclose(back[:, :, :cfg.nx], np.fft.irfft(R, cfg.nx, axis=2), atol=1e-13)
    assert np.all(back[:, :, cfg.nx:] == 0)


def test_dpdz_exact_on_polynomials():
    cfg = cf.Config(nx=8, ny=2, nzloc=9, nsubd=3, dt=1e-3, zlen=1.5,
                    z0=[0.0, 0.3, 0.9], zh=[0.3, 0.6, 0.6]).validate()
    o = Oracle(cfg)
    z = o.tables()["z"]
    f = np.zeros((cfg.nz, cfg.ny, cfg.nxpp))
    f[:] = (z ** 5)[:, None, None]
    df = o.dpdz(f)
    assert np.allclose(df, (5 * z ** 4)[:, None, None], atol=1e-10)


def test_filter_identity_for_low_modes():
    cfg = cf.Config(nx=8, ny=2, nzloc=9, nsubd=2, dt=1e-3, amp=36.0, p=4.0, pf=4.0).validate()
    o = Oracle(cfg)
    t = o.tables()
    assert t["sigma"][0] == 1.0 and abs(t["sigma"][-1] - math.exp(-36.0)) < 1e-30
    f = np.zeros((cfg.nz, cfg.ny, cfg.nxpp))
    f[:, 0, 0] = 1.0  # mean mode, constant in z
    g = o.filter3d(f)
    assert np.allclose(g, f, atol=1e-14)


@pytest.mark.parametrize("variant,tol", [(cf.IW_BC_NOSLIP, 5e-4)])
def test_shipped_2d_trajectory(golden, variant, tol):
    ref = np.array(golden["uveltest"])
    cflr = np.array(golden["cfl"])
    o = Oracle(cf.shipped_2d(bc_variant=variant))
    for s in range(9):
        o.step(1)
        lm = o.last_maxcalc()
        assert abs(lm["probe"] - ref[s, 1:]).max() <= tol * max(1e-30, abs(ref[s, 1:]).max())
        # CFL in z (w) to 4 digits, located at the same (i,j,k)
        if s > 0:
            assert abs(lm["cfl"][2] - cflr[s, 9]) <= 3e-4 * cflr[s, 9]
            assert lm["cfl_idx"][8] == int(cflr[s, 12])


def test_freeslip_variant_differs(golden):
    """The shipped trajectory was made with calcuvwt_noslip.f."""
    ref = np.array(golden["uveltest"])
    errs = {}
    for v in (cf.IW_BC_FREESLIP, cf.IW_BC_NOSLIP):
        o = Oracle(cf.shipped_2d(bc_variant=v))
        for s in range(9):
            o.step(1)
        errs[v] = abs(o.last_maxcalc()["probe"][0] - ref[8, 1]) / abs(ref[8, 1])
    assert errs[cf.IW_BC_NOSLIP] < 0.05 * errs[cf.IW_BC_FREESLIP]


def test_oracle_deterministic_across_threads():
    import oracle as om
    cfg = cf.Config(nx=16, ny=16, nzloc=9, nsubd=3, dt=1e-3).validate()
    outs = []
    for th in (1, 4):
        om.set_threads(th)
        o = Oracle(cfg)
        o.init_mode1(0.05, 1e-4, 7)
        o.step(3)
        outs.append(o.state())
    om.set_threads(om.max_threads())
    assert np.array_equal(outs[0], outs[1])


def test_factor_cache_is_bit_identical():
    cfg = cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=1e-3).validate()
    st = []
    for cache in (False, True):
        o = Oracle(cfg, cache=cache)
        o.init_mode1(0.05, 1e-4, 11)
        o.step(4)
        st.append(o.state())
    assert np.array_equal(st[0], st[1])


# ---------------------------------------------------------------------------
# Adaptive time step (maxcalc, various.f:892-982)
# ---------------------------------------------------------------------------
def wave_omega(xlen, zlen, brunt):
    """main.f:341-346 (bruntz = brunt)."""
    pi2 = 8.0 * math.atan(1.0)
    kx, m = pi2 / xlen, pi2 / (2.0 * zlen)
    return brunt * kx / math.sqrt(kx * kx + m * m)


def replay_dt_run(rule, run):
    """Drive a dt rule with the recorded run's cflzmax at the start of every
    step (cflx was not logged: 0) and return the (t, dt) of every change."""
    om = wave_omega(run["xlen"], run["zlen"], run["brunt"])
    t, dt, out = 0.0, run["dtin"], []
    for cz in run["cflz"]:
        r = rule(0.0, cz, t, dt, om)
        if r is not None:
            dt = r[0]
            out.append((t, dt))
        t = t + dt
    return out


def test_wave_frequency_matches_recorded_run(golden):
    run = golden["dt_run"]
    assert abs(wave_omega(run["xlen"], run["zlen"], run["brunt"]) - run["omega"]) <= 1e-14 * run["omega"]


def test_oracle_dt_rule_replays_recorded_run(golden):
    """All 18 changes of the recorded 400-step run (14 increases while
    cflz < 0.1, then 4 decreases by 5/4 when cflz > 0.7), at the same t, with
    the same dt, and no others."""
    import oracle
    run = golden["dt_run"]
    got = replay_dt_run(oracle.dt_rule, run)
    assert len(got) == len(run["changes"]) == 18
    for (t, dt), (rt, rdt) in zip(got, run["changes"]):
        assert abs(t - rt) <= 1e-13 * rt
        assert abs(dt - rdt) <= 1e-14 * rdt


def test_oracle_dt_rule_branches():
    import oracle
    om = wave_omega(2 * math.pi, 1.0, 1.0)
    tlim = 8.0 * math.atan(1.0) / (om * 50.0)
    assert oracle.dt_rule(0.0, 0.05, 20.0, 1.0, om) is None  # int(t/dt) = 20
    assert oracle.dt_rule(0.0, 0.5, 30.0, 1.0, om) is None  # CFL inside the window
    assert oracle.dt_rule(0.0, 0.05, 2.1, 0.1, om) == (0.1 / 0.8, 0.8)
    assert oracle.dt_rule(0.2, 0.05, 2.1, 0.1, om) == (0.1 / 1.25, 1.25)  # cflx wins over cflz < 0.1
    assert oracle.dt_rule(0.0, 0.8, 2.1, 0.1, om) == (0.1 / 1.25, 1.25)
    dn, c = oracle.dt_rule(0.0, 0.05, 30.0 * tlim, 0.9 * tlim, om)  # capped at Tlim
    assert c == 0.9 * tlim / tlim and dn == 0.9 * tlim / c
    assert oracle.dt_rule(0.0, float("nan"), 30.0, 1.0, om) is None


def test_oracle_adaptive_schedule():
    """imaxcalc = 1: dt changes exactly where the rule says from the CFL
    numbers of each step's start.  The change step itself has idtstep = 1, so
    it already sets the next step's variable-step coefficients of
    (dt, dt, cdt dt) and ends the change (ivardt = 0, cdt = 1; main.f:760-775,
    846-852); the step after that sets SS3/BDF3 again."""
    import oracle
    cfg = cf.Config(nx=16, ny=16, nzloc=9, nsubd=3, dt=2e-3, imaxcalc=1).validate()
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-4, 7)
    om = wave_omega(cfg.xlen, cfg.zlen, cfg.brunt)
    changes = []
    for _ in range(34):
        t0, dt0 = o.scalars()[0], o.dt_state()["dt"]
        o.step(1)
        lm = o.last_maxcalc()
        r = oracle.dt_rule(lm["cfl"][0], lm["cfl"][2], t0, dt0, om)
        st = o.dt_state()
        s = o.scalars()
        if r is None:
            assert st["dt"] == dt0
        else:
            changes.append(o.scalars()[1])
            dt, cdt = r
            assert st["dt"] == dt and st["ivardt"] == 0 and st["idtstep"] == 1 and st["cdt"] == 1.0
            for k, name in enumerate(("abvar1", "abvar2", "abvar3", "bdfvar1", "bdfvar2", "bdfvar3", "bdfvarv")):
                assert s[2 + k] == multistep(name, dt, dt, cdt * dt)
            o.step(1)
            st, s = o.dt_state(), o.scalars()
            assert st["ivardt"] == 0 and st["dt"] == dt
            assert list(s[2:9]) == [3.0, -3.0, 1.0, 3.0, -1.5, 1.0 / 3.0, 11.0 / 6.0]
    assert len(changes) >= 2 and changes[0] in (22, 23)


def test_animation_dump_schedule_replays_recorded_run(golden):
    """solver.f:141-142: a dump when t - Tdump >= dtanim at the start of
    convec, Tdump = t.  Driven by the recorded run's time steps (the replay of
    its dt changes), Tdump = 0 at the start and dtanim = 1 (the run's log does
    not print dtanim; 1 is the value whose schedule this is), the rule gives
    the run's 328 dumps with their counters and times, and no others."""
    import oracle
    run = golden["dt_run"]
    om = wave_omega(run["xlen"], run["zlen"], run["brunt"])
    t, dt, tdump, n, got = 0.0, run["dtin"], 0.0, 0, []
    for step, cz in enumerate(run["cflz"], 1):
        r = oracle.dt_rule(0.0, cz, t, dt, om)
        if r is not None:
            dt = r[0]
        if t - tdump >= 1.0:
            tdump = t
            n += 1
            got.append((n, t, step))
        t = t + dt
    assert len(got) == len(run["anim_dumps"]) == 328
    for (n1, t1, _), (n2, t2) in zip(got, run["anim_dumps"]):
        assert n1 == n2 and abs(t1 - t2) <= 1e-13 * max(1.0, t2)
    # and the run's animdump.log lines (solver.f:212-215), character for character
    assert [oracle.animdump_line(t1, n1, s1) for (n1, t1, s1) in got] == run["animdump_log"]


def test_oracle_animation_dump_rows(tmp_path):
    """vortanimout layout: the ZONE header, nx*nz lines of (1x,6(F25.16,3x)),
    and the rows the reference reads with j = ny+1 (the next z-plane; past
    the last plane v, temp and the spectral un of COMMON /flow/)."""
    cfg = cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=2e-3).validate()
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-4, 3)
    o.set_animation(2.5e-3, str(tmp_path))
    o.step(1)  # t = 0: 0 - 0 >= dtanim is false
    assert not list(tmp_path.iterdir())
    o.step(1)  # t = dt: no
    # what convec sees: maxcalc's round trip P, then the mean of w removed
    pf = [o.horfft(o.horfft(o.state(0)[q].copy(), 1), -1) for q in range(4)]
    pf[2][:, 0, 0:2] = 0.0
    ph = [o.horfft(f, 1) for f in pf]
    un = o.state(1)[0]
    o.step(1)  # t = 2 dt >= dtanim: dump 1 of the state at the start of this step
    files = sorted(p.name for p in tmp_path.iterdir() if p.name != "animdump.log")
    assert files == ["vortanimout_00001.dat"]
    import oracle as om
    assert (tmp_path / "animdump.log").read_text() == om.animdump_line(2 * cfg.dt, 1, 3) + "\n"
    lines = open(tmp_path / files[0]).read().split("\n")[:-1]
    assert lines[0] == " ZONE F=POINT, I=%12d , J=%12d" % (cfg.nx, cfg.nz)
    assert len(lines) == 1 + cfg.nx * cfg.nz
    assert all(len(ln) == 1 + 6 * 28 for ln in lines[1:])
    vals = np.array([[float(ln[1 + 28 * c: 26 + 28 * c]) for c in range(6)] for ln in lines[1:]])
    vals = vals.reshape(cfg.nz, cfg.nx, 6)
    z = o.tables()["z"]
    rg = -cfg.rho0 * cfg.brunt ** 2 / cfg.grav
    for k in range(cfg.nz):
        if k + 1 < cfg.nz:
            u, w, t = ph[0][k + 1, 0, :cfg.nx], ph[2][k + 1, 0, :cfg.nx], ph[3][k + 1, 0, :cfg.nx]
        else:
            u, w, t = ph[1][0, 0, :cfg.nx], ph[3][0, 0, :cfg.nx], un[0, 0, :cfg.nx]
        # F25.16 rounds at 5e-17
        assert np.allclose(vals[k, :, 1], z[k], rtol=0, atol=1e-16)
        for col, ref in ((2, u), (3, w), (4, t), (5, t + 1 + rg * z[k])):
            assert np.allclose(vals[k, :, col], ref, rtol=0, atol=1e-15 * max(1.0, np.abs(ref).max())), (k, col)


def test_mean_density_profile_matches_rhomean_dat(golden):
    """setup.f:170-184 of the shipped run wrote, from the top level down,
    z, rhomean(z), rhograd and (N(z)/N)^2 (6 digits each; the fifth column,
    fshear, enters the path only times fcshear = 0)."""
    rows = np.array(golden["rhomean"])
    o = Oracle(cf.shipped_2d())
    z = o.tables()["z"]
    assert rows.shape == (len(z), 5)
    for r, k in enumerate(range(len(z) - 1, -1, -1)):
        zz, rm, rg, n2 = rows[r, :4]
        assert abs(zz - z[k]) <= 5e-6 * max(abs(z[k]), 1e-2) + 1e-7
        assert abs(rm - o.rhomean(z[k])) <= 5e-6 * abs(o.rhomean(z[k]))
        assert abs(rg - o.rhograd()) <= 5e-6 * abs(o.rhograd())
        assert n2 == 1.0


def recorded_run_config(golden):
    """The recorded 400-step run (its log `output` and dtchange.dat): grid
    128 x (10 x 25) on runfolder/subd.dat, the namelist its log prints, the
    forced free-slip path (calcuvwt.f), maxcalc's adaptive step, zero initial
    fields.  fwave is not printed; the log shows the forcing at 1 for all 400
    steps, which any fwave >= 4.3 wave periods gives (input.dat's 8 is used)."""
    run = golden["dt_run"]
    p = run["params"]
    nx, nz = run["grid"]
    ns = run["nsubd"]
    sub = golden["subd_runfolder"][1:1 + ns]
    return cf.Config(nx=nx, ny=1, nzloc=nz // ns, nsubd=ns, dt=run["dtin"], xlen=run["xlen"], ylen=p["ylen"],
                     zlen=run["zlen"], brunt=run["brunt"], xnu=p["xnu"], xkappa=p["xkappa"], grav=p["grav"],
                     rho0=p["rho0"], umax=p["umax"], xacrit=p["xacrit"], xbcrit=p["xbcrit"], zcen=p["zcen"], fwave=8.0,
                     amp=p["amp"], p=p["p"], pf=p["pf"], fackc=p["fackc"], facdir=p["facdir"], facneumn=p["facneumn"],
                     facrobin=p["facrobin"], ispecfilternl=int(p["ispecfilternl"]),
                     ispecfilterexp=int(p["ispecfilterexp"]), nspecfilterexp=int(p["nspecfilterexp"]),
                     navgintrfc=int(p["navgintrfc"]), bc_variant=cf.IW_BC_FREESLIP, meanu_damping=1,
                     forcing=cf.IW_PADDLE_ABOVE_BOTTOM,
                     imaxcalc=1, z0=[r[0] for r in sub], zh=[r[1] for r in sub]).validate()


def recorded_dt_per_step(golden):
    """dt in effect at each of the recorded run's steps, from dtchange.dat."""
    run = golden["dt_run"]
    ch = {round(t, 9): dt for t, dt in run["changes"]}
    t, dt, out = 0.0, run["dtin"], []
    for _ in run["cflz"]:
        dt = ch.get(round(t, 9), dt)
        out.append(dt)
        t = t + dt
    return out


def probe_scale(rows, n, half=10):
    """Scale of the probe values near step n: the largest |value| of that
    probe within +-half steps (a probe crossing zero keeps the scale of its
    swing, so a relative bound means something there too)."""
    lo, hi = max(0, n - half), min(len(rows), n + half + 1)
    return np.abs(np.array([r[1:] for r in rows[lo:hi]])).max(axis=0)


def test_oracle_reproduces_recorded_run(golden):
    """The oracle on the recorded run's configuration, for all 400 steps:
    * maxcalc's cflz at the start of every step matches the run's log (16
      printed digits) to 1e-9 relative;
    * the probes u(32,1,10) and u(32,1,50) that maxcalc appends to
      uveltest.dat (rows 641-1040, 16 digits) match to 1e-9 of their scale;
    * dt changes at the same steps to the same values (to dtchange.dat's 15
      printed digits), decreases included.
    The agreement grows from 1e-13 over the first steps to about 1e-10 at the
    end: FP64 rounding differences carried through 400 steps."""
    import oracle
    run = golden["dt_run"]
    rows = golden["uveltest_recorded_run"]
    cfg = recorded_run_config(golden)
    dts = recorded_dt_per_step(golden)
    oracle.set_threads(oracle.max_threads())
    o = Oracle(cfg)
    assert len(rows) == len(run["cflz"]) == 400
    for n, (cz, dt) in enumerate(zip(run["cflz"], dts)):
        assert abs(o.scalars()[0] - rows[n][0]) <= 1e-13 * max(1.0, rows[n][0])  # t at the step's start
        o.step(1)
        lm = o.last_maxcalc()
        c = lm["cfl"][2]
        assert abs(c - cz) <= 1e-9 * cz or (cz == 0.0 and c == 0.0), (n + 1, c, cz)
        assert np.all(np.abs(lm["probe"] - np.array(rows[n][1:])) <= 1e-9 * probe_scale(rows, n) + 1e-300), \
            (n + 1, lm["probe"], rows[n])
        assert abs(o.dt_state()["dt"] - dt) <= 1e-14 * dt, (n + 1, o.dt_state()["dt"], dt)  # 15 printed digits


def test_recorded_run_paddle_leaves_out_the_bottom_point(golden):
    """The one difference between the shipped solver.f and the binary that
    made the recorded run: the paddle loop of solver.f:848 runs over
    k = 1..nz, while its comment says the bottom point is overlooked.  Over
    the first 6 steps, the paddle on every level (IW_PADDLE_ALL_LEVELS) puts
    the probes 2e-5 to 4e-4 and cflz 1e-4 away from the recorded values;
    leaving the bottom point out (IW_PADDLE_ABOVE_BOTTOM) brings both within
    1e-12."""
    run = golden["dt_run"]
    rows = golden["uveltest_recorded_run"]
    errs = {}
    for mode in (cf.IW_PADDLE_ALL_LEVELS, cf.IW_PADDLE_ABOVE_BOTTOM):
        o = Oracle(recorded_run_config(golden).replace(forcing=mode))
        ep, ec = 0.0, 0.0
        for n in range(6):
            o.step(1)
            lm = o.last_maxcalc()
            if n:
                ep = max(ep, float(np.max(np.abs(lm["probe"] - rows[n][1:]) / np.abs(rows[n][1:]))))
                ec = max(ec, abs(lm["cfl"][2] - run["cflz"][n]) / run["cflz"][n])
        errs[mode] = (ep, ec)
    assert errs[cf.IW_PADDLE_ALL_LEVELS][0] > 1e-4 and errs[cf.IW_PADDLE_ALL_LEVELS][1] > 5e-5
    assert errs[cf.IW_PADDLE_ABOVE_BOTTOM][0] < 1e-12 and errs[cf.IW_PADDLE_ABOVE_BOTTOM][1] < 1e-12
