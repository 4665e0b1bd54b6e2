"""Field dumps (iw_write_fields: plotf, output.f:118-265) through the C ABI
against the oracle's plotf.

* iform 0: headers and grids equal; REAL*4 fields equal up to one float ulp
  (the GPU and oracle physical values agree to ~1e-15 before rounding).
* iform 1: the same text layout; values equal up to one unit of the 6th digit.
* Asynchronous dumps: steps taken while the file is written do not change
  it; a mixed-precision handle dumps its FP32 fields; an unwritable path is
  reported by iw_wait_fields.
"""
import numpy as np
import pytest

from iwrepo_b200 import config as cf
from test_field_output import parse_formatted, parse_unformatted

pytestmark = pytest.mark.gpu


def _pair(precision=cf.IW_PREC_FP64):
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = cf.Config(nx=32, ny=16, nzloc=9, nsubd=3, dt=2e-3, precision=precision).validate()
    o, s = Oracle(cfg), iw.Solver(cfg)
    o.init_mode1(0.05, 1e-4, 4)
    o.step(3)
    s.set_state(*[o.state(lv) for lv in range(5)], t=o.scalars()[0], istep=3)
    return cfg, o, s


def test_unformatted_dump_equals_oracle(tmp_path):
    cfg, o, s = _pair()
    o.plotf(tmp_path / "o.dat", 0)
    s.write_fields(tmp_path / "s.dat", 0)
    to, do, xo, yo, zo, fo = parse_unformatted(tmp_path / "o.dat", cfg)
    ts, ds, xs, ys, zs, fs = parse_unformatted(tmp_path / "s.dat", cfg)
    assert ts == to and ds == do
    for a, b in ((xs, xo), (ys, yo), (zs, zo)):
        assert np.abs(a - b).max() <= 1e-15 * max(1.0, np.abs(b).max())
    assert np.all(np.abs(fs - fo) <= np.spacing(np.abs(fo).astype(np.float32)))
    assert not fs[..., cfg.nx:].any()
    s.close()


def test_formatted_dump_equals_oracle(tmp_path):
    cfg, o, s = _pair()
    o.plotf(tmp_path / "o.txt", 1)
    s.write_fields(tmp_path / "s.txt", 1)
    do, vo, lo = parse_formatted(tmp_path / "o.txt", cfg)
    ds, vs, ls = parse_formatted(tmp_path / "s.txt", cfg)
    assert do == ds and [len(x) for x in lo] == [len(x) for x in ls]
    vo, vs = np.array(vo), np.array(vs)
    assert np.all(np.abs(vs - vo) <= 1.0001e-5 * np.abs(vo) + 1e-300)
    assert np.mean(vs == vo) > 0.999  # text differs only where the 6th digit is a rounding tie
    s.close()


def test_async_dump_is_the_state_at_the_call(tmp_path):
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=32, ny=16, nzloc=9, nsubd=3, dt=2e-3).validate()
    a, b = iw.Solver(cfg), iw.Solver(cfg)
    for x in (a, b):
        x.init_mode1(0.05, 1e-4, 6)
        x.step(2)
    a.write_fields(tmp_path / "async.dat", 0, wait=False)
    a.step(3)
    a.wait_fields()
    b.write_fields(tmp_path / "sync.dat", 0)
    assert (tmp_path / "async.dat").read_bytes() == (tmp_path / "sync.dat").read_bytes()
    b.step(3)
    assert np.array_equal(a.state(0), b.state(0))
    a.write_fields(tmp_path / "missing_dir" / "x.dat", 0, wait=False)
    with pytest.raises(iw.IwError, match="cannot open"):
        a.wait_fields()
    a.close()
    b.close()


def test_mixed_precision_dump(tmp_path):
    cfg, o, s = _pair(cf.IW_PREC_MIXED)
    o.plotf(tmp_path / "o.dat", 0)
    s.write_fields(tmp_path / "s.dat", 0)
    fo = parse_unformatted(tmp_path / "o.dat", cfg)[5]
    fs = parse_unformatted(tmp_path / "s.dat", cfg)[5]
    for q in range(4):
        assert np.linalg.norm(fs[q] - fo[q]) <= 1e-6 * np.linalg.norm(fo[q]), q
    s.close()
