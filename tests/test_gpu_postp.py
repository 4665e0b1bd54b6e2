"""TKE budget through the C ABI (iw_postp, iw_set_postp: postp.f:9-70 and
415-732) against the oracle's postp.

* iw_postp on the oracle's state: every value within 1e-10 (the production
  terms with a floor of 1e-12 of their scale).
* iw_set_postp: energy.dat, energy_wake.dat and wakescale.dat get the
  reference's headers and one line every npostp steps, FORMAT
  (1x,F10.4,17(2x,E12.6)) / (1x,F10.4,8(2x,E12.6)), values as the oracle's
  postp after the same steps to the printed digits.
* A mixed-precision handle: the energetic terms within 1e-5.
"""
import numpy as np
import pytest

from iwrepo_b200 import config as cf

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    return cf.Config(nx=32, ny=16, nzloc=9, nsubd=3, dt=2e-3, ylen=3.0, **kw).validate()


def _close(a, b, tol, floor=0.0):
    return np.all(np.abs(np.asarray(a) - np.asarray(b)) <= tol * np.abs(b) + floor)


def _oracle_after(cfg, nsteps):
    from oracle import Oracle
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-3, 5)
    o.step(nsteps)
    return o


def test_postp_equals_oracle():
    import iwrepo_b200 as iw
    cfg = _cfg()
    o = _oracle_after(cfg, 3)
    s = iw.Solver(cfg)
    s.set_state(*[o.state(lv) for lv in range(5)], t=o.scalars()[0], istep=3)
    s.set_postp(0, 0.001)  # tstart only
    e, w = s.postp()
    eo, wo = o.postp(tstart=0.001)
    scale = max(abs(eo[6]), abs(eo[7]))
    for n in range(18):
        floor = 1e-12 * scale if n in (6, 7, 8) else 0.0
        assert _close(e[n], eo[n], 1e-10, floor), (n, e[n], eo[n])
    assert _close(w, wo, 1e-10)
    s.close()


def _parse(path, nval):
    lines = open(path).read().split("\n")[:-1]
    head, rows = lines[0], []
    for ln in lines[1:]:
        assert len(ln) == 11 + 14 * (nval - 1), repr(ln)
        rows.append([float(ln[1:11])] + [float(ln[13 + 14 * c: 25 + 14 * c]) for c in range(nval - 1)])
    return head, np.array(rows)


def test_postp_files(tmp_path):
    import iwrepo_b200 as iw
    cfg = _cfg()
    s = iw.Solver(cfg)
    s.init_mode1(0.05, 1e-3, 5)
    s.set_postp(2, 0.0, str(tmp_path))
    s.run(4, graph=True)
    want = [_oracle_after(cfg, n).postp() for n in (2, 4)]
    head, rows = _parse(tmp_path / "energy.dat", 18)
    assert head.startswith(' VARIABLES ="TIME","Nt","TKE","u1tke"') and head.endswith('"TKEmean","Tvar"')
    assert rows.shape == (2, 18)
    for r, (e, _) in zip(rows, want):
        assert abs(r[0] - e[0]) <= 5e-5 and _close(r[1:], e[1:], 1.0001e-5, 1e-12 * np.abs(e[1:]).max())
    head, rows = _parse(tmp_path / "energy_wake.dat", 18)
    for r, (_, wv) in zip(rows, want):
        assert _close(r[1:], wv[1:], 1.0001e-5, 1e-300) and not np.any(r[2:16])
    head, rows = _parse(tmp_path / "wakescale.dat", 9)
    assert head == ' VARIABLES ="TIME","Nt","umax","umaxy","umaxz","L_y","L_z","yc","zc"'
    assert rows.shape == (2, 9) and not np.any(rows[:, 2:])
    s.close()


def test_postp_mixed_precision():
    import iwrepo_b200 as iw
    cfg = _cfg()
    o = _oracle_after(cfg, 3)
    s = iw.Solver(cfg.replace(precision=cf.IW_PREC_MIXED))
    s.set_state(*[o.state(lv) for lv in range(5)], t=o.scalars()[0], istep=3)
    e, _ = s.postp()
    eo, _ = o.postp()
    for n in (2, 3, 4, 5, 10, 13, 16, 17):  # tketot, u1..u3tke, epsilon, chi, tkemean, tempvar
        assert _close(e[n], eo[n], 1e-5), (n, e[n], eo[n])
    s.close()
