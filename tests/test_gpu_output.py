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


def test_animation_dumps_equal_oracle(tmp_path):
    """convec's animation dumps (iw_set_animation, solver.f:136-222): the same
    files at the same steps as the oracle's, the same header and layout,
    values to 1e-12 of each column's scale (the rows the reference reads with
    j = ny+1 included).  Requested graph replay stays eager while dumps are on."""
    import iwrepo_b200 as iw
    from oracle import Oracle
    cfg = cf.Config(nx=32, ny=16, nzloc=9, nsubd=3, dt=2e-3).validate()
    o, s = Oracle(cfg), iw.Solver(cfg)
    (tmp_path / "o").mkdir()
    (tmp_path / "s").mkdir()
    for x, d in ((o, "o"), (s, "s")):
        x.init_mode1(0.05, 1e-4, 9)
        x.set_animation(3.5e-3, str(tmp_path / d))
    o.step(9)
    s.run(9, graph=True)
    s.wait_fields()
    names = sorted(p.name for p in (tmp_path / "o").iterdir() if p.name != "animdump.log")
    assert names == sorted(p.name for p in (tmp_path / "s").iterdir() if p.name != "animdump.log")
    assert names == ["vortanimout_%05d.dat" % n for n in (1, 2, 3, 4)]  # t = 2, 4, 6, 8 dt
    log = (tmp_path / "s" / "animdump.log").read_text()
    assert log == (tmp_path / "o" / "animdump.log").read_text() and len(log.splitlines()) == 4
    for n in names:
        lo = open(tmp_path / "o" / n).read().split("\n")
        ls = open(tmp_path / "s" / n).read().split("\n")
        assert lo[0] == ls[0] and len(lo) == len(ls) == cfg.nx * cfg.nz + 2
        assert [len(x) for x in lo] == [len(x) for x in ls]
        vo = np.array([[float(ln[1 + 28 * c: 26 + 28 * c]) for c in range(6)] for ln in lo[1:-1]])
        vs = np.array([[float(ln[1 + 28 * c: 26 + 28 * c]) for c in range(6)] for ln in ls[1:-1]])
        for c in range(6):
            assert np.abs(vs[:, c] - vo[:, c]).max() <= 1e-12 * max(1e-300, np.abs(vo[:, c]).max()), (n, c)
    a = s.state()
    b = o.state()  # the steps themselves: the full-step FP64 bar
    assert max(np.linalg.norm(a[q] - b[q]) / np.linalg.norm(b[q]) for q in range(4)) <= 1e-10
    s.close()


def test_legendre_spectra_equal_oracle(tmp_path):
    """speclegencalc every 3 steps (iw_set_speclegen): the same files as the
    oracle's, values equal up to the 6th digit (and a round-off floor for the
    top modes); ny = 1 is refused."""
    import iwrepo_b200 as iw
    from oracle import Oracle
    from test_field_output import parse_speclegen
    cfg = cf.Config(nx=32, ny=16, nzloc=9, nsubd=3, dt=2e-3).validate()
    o, s = Oracle(cfg), iw.Solver(cfg)
    (tmp_path / "o").mkdir()
    (tmp_path / "s").mkdir()
    for x, d in ((o, "o"), (s, "s")):
        x.init_mode1(0.05, 1e-4, 2)
        x.set_speclegen(3, str(tmp_path / d))
    o.step(7)
    s.run(7, graph=True)
    s.wait_fields()
    names = sorted(p.name for p in (tmp_path / "o").iterdir())
    assert names == sorted(p.name for p in (tmp_path / "s").iterdir())
    assert names == sorted("speclegen%s%s.dat" % (c, t) for c in "uvwT" for t in ("0.006", "0.012"))
    for n in names:
        a, b = parse_speclegen(tmp_path / "s" / n, cfg.nsubd), parse_speclegen(tmp_path / "o" / n, cfg.nsubd)
        assert np.all(np.abs(a - b) <= 1.0001e-5 * np.abs(b) + 1e-12 * np.abs(b).max()), n
    # the dumps leave the steps alone: the state equals the oracle's
    a, b = s.state(), o.state()
    assert max(np.linalg.norm(a[q] - b[q]) / np.linalg.norm(b[q]) for q in range(4)) <= 1e-10
    flat = cf.Config(nx=32, ny=1, nzloc=9, nsubd=3, dt=2e-3).validate()
    f = iw.Solver(flat)
    with pytest.raises(iw.IwError, match="ny >= 2"):
        f.set_speclegen(3, str(tmp_path))
    for x in (s, f):
        x.close()
