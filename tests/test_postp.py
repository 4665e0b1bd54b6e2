"""TKE budget (postp, postp.f:9-70 and 415-732) on the CPU: the oracle's
values against numpy from the oracle's own physical fields.

* umean = x mean of u on levels 2..nz (0 at level 1); u' = u - umean;
* tketot, u1/u2/u3tke, tempvar, tkemean as sums over levels 2..nz;
* prodz with d(umean)/dz from the subdomain derivative matrix, prody with
  d(umean)/dy from numpy's real FFT (Nyquist term dropped);
* bflux = 0 (ra = 0), the subgrid terms 0, epstot = epsilon, chitot = chi;
* the wake line: zeros but the times and tkemean.
"""
import numpy as np

from iwrepo_b200 import config as cf
from oracle import Oracle


def _state(ny=8):
    cfg = cf.Config(nx=16, ny=ny, nzloc=9, nsubd=3, dt=2e-3, ylen=3.0).validate()
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-3, 5)
    o.step(3)
    return cfg, o


def _numpy_budget(o, cfg):
    st = o.state(0)
    ph = [o.horfft(st[q].copy(), 1) for q in range(4)]   # (nz, ny, nxpp), padding 0
    um = ph[0][..., :cfg.nx].mean(axis=2)
    um[0] = 0.0
    ph[0][..., :cfg.nx] -= um[..., None]
    # energycalc_postp transforms u', v, w, temp to spectral space and back
    # before its sums; in horfft's conventions that round trip is not the
    # identity (it rescales the x-Nyquist column)
    ph = [o.horfft(o.horfft(f, -1), 1)[..., :cfg.nx] for f in ph]
    up, v, w, t = ph
    sl = slice(1, None)
    tb = o.tables()
    N = cfg.nzloc
    dz = np.zeros_like(um)
    for ks in range(cfg.nsubd):
        dz[ks * N:(ks + 1) * N] = (2.0 / cfg.zh[ks]) * (tb["d"] @ um[ks * N:(ks + 1) * N])
    if cfg.ny > 1:
        c = np.fft.rfft(um, axis=1)
        ky = np.arange(c.shape[1]) * (2 * np.pi / cfg.ylen)
        c = c * 1j * ky
        c[:, -1] = 0.0
        dy = np.fft.irfft(c, n=cfg.ny, axis=1)
    else:
        dy = np.zeros_like(um)
    return dict(
        tketot=0.5 * np.sum(up[sl] ** 2 + v[sl] ** 2 + w[sl] ** 2),
        u1=np.sum(up[sl] ** 2), u2=np.sum(v[sl] ** 2), u3=np.sum(w[sl] ** 2),
        prody=-np.sum(dy[sl][..., None] * up[sl] * v[sl]),
        prodz=-np.sum(dz[sl][..., None] * up[sl] * w[sl]),
        tempvar=np.sum(t[sl] ** 2), tkemean=0.5 * cfg.nx * np.sum(um[sl] ** 2))


def _close(a, b, tol=1e-11, floor=0.0):
    return abs(a - b) <= tol * abs(b) + floor


def test_oracle_budget_against_numpy():
    cfg, o = _state()
    e, w = o.postp(tstart=0.001)
    ref = _numpy_budget(o, cfg)
    t = o.scalars()[0]
    assert e[0] == t - 0.001 and e[1] == (t - 0.001) * cfg.brunt
    scale = max(abs(e[6]), abs(e[7]), 1e-30)
    for k, n in (("tketot", 2), ("u1", 3), ("u2", 4), ("u3", 5), ("tempvar", 17), ("tkemean", 16)):
        assert _close(e[n], ref[k]), (k, e[n], ref[k])
    assert _close(e[6], ref["prody"], 1e-9, 1e-12 * scale) and _close(e[7], ref["prodz"], 1e-9, 1e-12 * scale)
    assert e[8] == e[6] + e[7]
    assert e[9] == 0.0 and e[11] == 0.0 and e[14] == 0.0      # bflux (ra = 0), epssgs, chisgs
    assert e[12] == e[10] and e[15] == e[13] and e[10] > 0 and e[13] > 0
    assert list(w[:2]) == list(e[:2]) and w[16] == e[16]
    assert not np.any(w[2:16]) and w[17] == 0.0


def test_oracle_budget_2d_has_no_y_production():
    cfg, o = _state(ny=1)
    e, _ = o.postp()
    ref = _numpy_budget(o, cfg)
    assert e[6] == 0.0 and _close(e[7], ref["prodz"], 1e-9, 1e-20)
