"""Restart files (output.f:2-117, restart.f:2-126, main.f:555-632) on the CPU
through the oracle.

* The file has output.f's 49 records in its order and sizes, in ifort's
  unformatted sequential framing, then the continuation record.
* t, pr, the dims and the state levels sit where restart.f reads them.
* Exact mode continues a run bit for bit; the reference's mode (istart = 1)
  gives main.f's coefficients for the first steps after the read.
* Bad files are refused without changing the state.
"""
import struct

import numpy as np
import pytest

from iwrepo_b200 import config as cf
from oracle import Oracle, multistep
from restart_format import extra, f8, layout, records, state_levels


def _cfg(**kw):
    return cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=2e-3, **kw).validate()


def _levels(o):
    return np.stack([o.state(lv) for lv in range(5)])


def test_oracle_file_follows_output_f(tmp_path):
    cfg = _cfg()
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-4, 3)
    o.step(4)
    p = tmp_path / "run.dat"
    o.write_restart(p)
    recs = records(p)
    lay = layout(cfg)
    assert len(recs) == len(lay) + 1
    for k, (n8, n4) in enumerate(lay):
        assert len(recs[k]) == 8 * n8 + 4 * n4, k + 1
    assert f8(recs[0])[0] == o.scalars()[0]                      # t
    assert tuple(f8(recs[1])) == (cfg.xnu, 0.0)                  # pr, ra
    assert struct.unpack("<9i", recs[2]) == (cfg.nx, cfg.ny, cfg.nz, cfg.nzloc - 1, cfg.nxpp * cfg.ny, cfg.ntot,
                                             cfg.nsubd, cfg.nzloc, 1)
    # (z0, zh, isubdtype) triples
    for k in range(cfg.nsubd):
        z0, zh, it = struct.unpack_from("<ddi", recs[10], 20 * k)
        assert (z0, zh, it) == (cfg.z0[k], cfg.zh[k], 1)
    assert f8(recs[22])[0] == cfg.umax
    assert np.array_equal(state_levels(recs, cfg), _levels(o))
    (istep, ivardt, idtstep, istart), dbl = extra(recs)
    assert (istep, ivardt, idtstep, istart) == (4, 0, 0, 0)
    assert dbl[0] == cfg.dt and list(dbl[2:]) == list(o.scalars()[2:9])


def test_oracle_exact_restart_continues_bit_for_bit(tmp_path):
    cfg = _cfg()
    a, b = Oracle(cfg), Oracle(cfg)
    a.init_mode1(0.05, 1e-4, 3)
    a.step(5)
    p = tmp_path / "run.dat"
    a.write_restart(p)
    b.read_restart(p, "exact")
    assert np.array_equal(_levels(a), _levels(b))
    assert np.array_equal(a.scalars(), b.scalars())
    a.step(4)
    b.step(4)
    assert np.array_equal(_levels(a), _levels(b))


def test_oracle_reference_restart_schedule(tmp_path):
    """main.f:613-632: the first step after the read uses the coefficients of a
    step dt after two of cdtin*dt; it sets (dt, dt, cdtin*dt) for the second
    (main.f:716-730, 820-826); from the third on SS3/BDF3."""
    cfg = _cfg()
    a, b = Oracle(cfg), Oracle(cfg)
    a.init_mode1(0.05, 1e-4, 3)
    a.step(5)
    p = tmp_path / "run.dat"
    a.write_restart(p)
    dt, cdt = cfg.dt, 1.25
    b.read_restart(p, "reference", cdtin=cdt)
    s = b.scalars()
    assert s[0] == a.scalars()[0] and s[1] == 0
    names = ("abvar1", "abvar2", "abvar3", "bdfvar1", "bdfvar2", "bdfvar3", "bdfvarv")
    assert list(s[2:9]) == [multistep(n, dt, cdt * dt, cdt * dt) for n in names]
    b.step(1)
    assert list(b.scalars()[2:9]) == [multistep(n, dt, dt, cdt * dt) for n in names]
    assert b.dt_state()["cdt"] == cdt
    b.step(1)
    assert list(b.scalars()[2:9]) == [3.0, -3.0, 1.0, 3.0, -1.5, 1.0 / 3.0, 11.0 / 6.0]
    assert np.all(np.isfinite(b.state(0)))


def test_oracle_refuses_bad_files(tmp_path):
    cfg = _cfg()
    a = Oracle(cfg)
    a.init_mode1(0.05, 1e-4, 3)
    a.step(3)
    p = tmp_path / "run.dat"
    a.write_restart(p)
    raw = p.read_bytes()
    b = Oracle(cfg)
    b.init_mode1(0.01, 0.0, 9)
    before = _levels(b)
    # truncated inside a field record
    (tmp_path / "cut.dat").write_bytes(raw[:len(raw) // 2])
    with pytest.raises(RuntimeError):
        b.read_restart(tmp_path / "cut.dat", "reference")
    # the reference's own files end after record 49: fine for the reference's
    # mode, refused for exact continuation
    recs = records(p)
    body = b"".join(struct.pack("<i", len(r)) + r + struct.pack("<i", len(r)) for r in recs[:49])
    (tmp_path / "ref.dat").write_bytes(body)
    with pytest.raises(RuntimeError):
        b.read_restart(tmp_path / "ref.dat", "exact")
    assert np.array_equal(_levels(b), before)
    b.read_restart(tmp_path / "ref.dat", "reference")
    assert np.array_equal(_levels(b), _levels(a))
    # other dims
    c = Oracle(_cfg().replace(nx=32))
    with pytest.raises(RuntimeError):
        c.read_restart(p, "reference")
