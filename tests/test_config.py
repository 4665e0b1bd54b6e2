"""Host-side configuration: namelists, subd.dat, validation of what the
reference leaves unchecked."""
import math

import pytest

from iwrepo_b200 import config as cf

INPUT_DAT = """ $inputs
   istart = 0,
   dtin = 0.1,
   nsteps = 400,
   cdtin = 1.0,
   fwave = 8.0 $
 $params
    xlen = 20.0, ylen = 1., zlen = 5.0, brunt = 0.2,
    xnu = 1.e-5, xkappa = 1.e-5, grav = 9.81, expan = 3.38e-3,
    umax = 0.01, rho0 = 1.e3, xacrit = 2.5, xbcrit = 0.84, zcen = 0.13 $
$mflags
    irelax = 0, ispecfilternl = 1, ispecfilterexp = 1, nspecfilterexp =1,
    amp = 35., p = 5.0, pf = 10.0, fackc = 0., facdir = 1.e0, facneumn = 1.e0,
    facrobin  = 1.e4, navgintrfc = 1 $
"""
SUBD_DAT = "3\n0.0 1.0\n1.0 2.5\n3.5 1.5\n"


def test_namelists(tmp_path):
    (tmp_path / "input.dat").write_text(INPUT_DAT)
    (tmp_path / "subd.dat").write_text(SUBD_DAT)
    c = cf.from_files(str(tmp_path / "input.dat"), str(tmp_path / "subd.dat"), nx=16, ny=1, nzloc=9, nsubd=3)
    assert c.dt == 0.1 and c.xlen == 20.0 and c.brunt == 0.2 and c.facrobin == 1e4
    assert c.amp == 35.0 and c.p == 5.0 and c.pf == 10.0 and c.forcing == cf.IW_PADDLE_ALL_LEVELS
    assert c.zh == [1.0, 2.5, 1.5] and c.nz == 27


@pytest.mark.parametrize("kw,msg", [
    (dict(nx=14 * 7), "nx"), (dict(nx=15), "nx"), (dict(ny=6 * 7), "ny"), (dict(nzloc=2), "nzloc"),
    (dict(nsubd=0), "nsubd"), (dict(dt=-1.0), "dt"), (dict(xnu=0.0), "xnu"),
])
def test_invalid_dims(kw, msg):
    base = dict(nx=16, ny=8, nzloc=9, nsubd=3, dt=1e-3)
    base.update(kw)
    with pytest.raises(cf.ConfigError, match=msg):
        cf.Config(**base).validate()


def test_invalid_subdomain_tables():
    with pytest.raises(cf.ConfigError):
        cf.Config(nx=16, ny=8, nzloc=9, nsubd=2, dt=1e-3, z0=[0.0, 0.4], zh=[0.5, 0.5]).validate()
    with pytest.raises(cf.ConfigError):
        cf.Config(nx=16, ny=8, nzloc=9, nsubd=2, dt=1e-3, z0=[0.0, 0.5], zh=[0.5, -0.5]).validate()
    with pytest.raises(cf.ConfigError):
        cf.parse_subd("4\n0 1\n1 1\n")


def test_baselines():
    c0 = cf.baseline("C0")
    assert (c0.nx, c0.ny, c0.nz, c0.dt) == (64, 64, 68, 1e-3) and abs(1 / c0.xnu - 1000) < 1e-9
    c3 = cf.baseline("C3")
    assert (c3.nx, c3.nsubd, c3.nzloc) == (512, 12, 33) and c3.grid_points == 512 * 512 * 396
    members = cf.ensemble_members(48)
    assert len(members) == 48
    for m in members:
        assert m.nx in (64, 96, 128, 192) and 3 <= m.nsubd <= 8 and 17 <= m.nzloc <= 25
        assert 1000 <= 1 / m.xnu <= 5000 and 0.01 <= m.member_amp <= 0.1


def test_c_structs_roundtrip():
    c = cf.shipped_2d()
    p = c.c_params()
    assert p.zh[11] == 0.225 and p.xacrit == 2.5 and p.bc_variant == cf.IW_BC_FREESLIP
    d = c.c_dims()
    assert (d.nx, d.ny, d.nzloc, d.nsubd) == (256, 1, 25, 12)
