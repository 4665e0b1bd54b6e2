"""Restart files through the C ABI (iw_write_restart, iw_read_restart) against
the oracle's writer and reader.

* The library's file equals the oracle's for the same state: framing, sizes,
  the scalars and the 20 field records bit for bit, the setup tables to 1e-13.
* Exact mode continues a run bit for bit (FP64 and mixed precision).
* The reference's mode (main.f istart = 1) on a file the oracle wrote: the
  following steps agree with the oracle doing the same to 1e-10.
* A file of other dims is refused and leaves the state as it was.
"""
import struct

import numpy as np
import pytest

from iwrepo_b200 import config as cf
from restart_format import f8, layout, records

pytestmark = pytest.mark.gpu


def rel(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def _cfg(**kw):
    return cf.Config(nx=32, ny=16, nzloc=9, nsubd=3, dt=2e-3, **kw).validate()


def _levels(s):
    return np.stack([s.state(lv) for lv in range(5)])


def test_library_file_equals_oracle_file(tmp_path):
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = _cfg()
    o, s = Oracle(cfg), iw.Solver(cfg)
    o.init_mode1(0.05, 1e-4, 3)
    o.step(3)
    lev = [o.state(lv) for lv in range(5)]
    s.set_state(*lev, t=o.scalars()[0], istep=3)
    o.write_restart(tmp_path / "o.dat")
    s.write_restart(tmp_path / "s.dat")
    ro, rs = records(tmp_path / "o.dat"), records(tmp_path / "s.dat")
    assert len(ro) == len(rs) == len(layout(cfg)) + 1
    for k in range(49):
        assert len(ro[k]) == len(rs[k]), k + 1
        if k in (2, 10):  # records holding INTEGER items
            assert ro[k] == rs[k], k + 1
        elif 3 <= k <= 21:  # setup tables
            a, b = f8(rs[k]), f8(ro[k])
            assert np.abs(a - b).max() <= 1e-13 * max(1.0, np.abs(b).max()), k + 1
        else:
            assert ro[k] == rs[k], k + 1
    s.close()


@pytest.mark.parametrize("precision", [cf.IW_PREC_FP64, cf.IW_PREC_MIXED])
def test_exact_restart_continues_bit_for_bit(tmp_path, precision):
    import iwrepo_b200 as iw
    cfg = _cfg(precision=precision)
    a, b, c = iw.Solver(cfg), iw.Solver(cfg), iw.Solver(cfg)
    for x in (a, b):
        x.init_mode1(0.05, 1e-4, 8)
    a.step(11)
    b.step(6)
    b.write_restart(tmp_path / "run.dat")
    c.read_restart(tmp_path / "run.dat", "exact")
    c.step(5)
    assert np.array_equal(_levels(a), _levels(c))
    assert a.diag()["t"] == c.diag()["t"] and a.diag()["istep"] == c.diag()["istep"] == 11
    for x in (a, b, c):
        x.close()


def test_reference_restart_matches_oracle(tmp_path):
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = _cfg()
    w = Oracle(cfg)
    w.init_mode1(0.05, 1e-4, 12)
    w.step(6)
    w.write_restart(tmp_path / "run.dat")
    o, s = Oracle(cfg), iw.Solver(cfg)
    o.read_restart(tmp_path / "run.dat", "reference", cdtin=1.25)
    s.read_restart(tmp_path / "run.dat", "reference", cdtin=1.25)
    o.step(8)
    s.step(8)
    a, b = s.state(), o.state()
    for q in range(4):
        assert rel(a[q], b[q]) <= 1e-10, q
    assert s.diag()["istep"] == 8
    s.close()


def test_restart_of_other_dims_is_refused(tmp_path):
    import iwrepo_b200 as iw
    small, big = _cfg(), _cfg().replace(nx=64)
    a, b = iw.Solver(small), iw.Solver(big)
    a.init_mode1(0.05, 1e-4, 1)
    b.init_mode1(0.02, 1e-4, 2)
    a.write_restart(tmp_path / "run.dat")
    before = _levels(b)
    with pytest.raises(iw.IwError, match="record"):
        b.read_restart(tmp_path / "run.dat", "reference")
    with pytest.raises(iw.IwError):
        b.read_restart(tmp_path / "absent.dat", "reference")
    assert np.array_equal(_levels(b), before)
    raw = (tmp_path / "run.dat").read_bytes()
    recs = records(tmp_path / "run.dat")
    ref_only = b"".join(struct.pack("<i", len(r)) + r + struct.pack("<i", len(r)) for r in recs[:49])
    (tmp_path / "ref.dat").write_bytes(ref_only)
    c = iw.Solver(small)
    with pytest.raises(iw.IwError, match="continuation"):
        c.read_restart(tmp_path / "ref.dat", "exact")
    c.read_restart(tmp_path / "ref.dat", "reference")
    assert np.array_equal(c.state(0), a.state(0)) and len(raw) > len(ref_only)
    for x in (a, b, c):
        x.close()


def test_read_restart_restarts_the_animation_counter(tmp_path):
    """Tdump and the dump counter are not in the file (restart.f does not read
    them): after a read they start from 0, as in a restarted reference run."""
    import iwrepo_b200 as iw
    cfg = _cfg()
    a = iw.Solver(cfg)
    a.init_mode1(0.05, 1e-4, 4)
    d = tmp_path / "anim"
    d.mkdir()
    a.set_animation(1.5 * cfg.dt, str(d))
    a.step(5)  # dumps at t = 2 dt and 4 dt
    a.wait_fields()
    assert sorted(p.name for p in d.iterdir()) == ["animdump.log", "vortanimout_00001.dat", "vortanimout_00002.dat"]
    a.write_restart(tmp_path / "run.dat")
    for p in list(d.iterdir()):
        p.unlink()
    a.read_restart(tmp_path / "run.dat", "reference")
    a.step(1)  # t - Tdump = 5 dt - 0 >= dtanim: dump number 1 again
    a.wait_fields()
    assert sorted(p.name for p in d.iterdir()) == ["animdump.log", "vortanimout_00001.dat"]
    a.close()
