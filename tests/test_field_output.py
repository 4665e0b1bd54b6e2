"""Field dumps (plotf, output.f:118-265) on the CPU through the oracle.

* iform 0: t | nx ny nz ntot | x | y | z | u v w temp as REAL*4 in physical
  space, in ifort's unformatted framing; the fields equal the inverse
  horfft of the state rounded to REAL*4, padding entries 0.
* iform 1: FORMAT 5e14.6 / 5i10 text: 14-character fields, 5 per line, the
  four fields as one list; values within the rounding of 6 digits (5e-6).
* The Ew.d formatter itself on known cases (mantissa 0.dddddd, carries,
  negative exponents, zero).
"""
import math
import struct

import numpy as np

from iwrepo_b200 import config as cf
from oracle import Oracle
from restart_format import records


def _oracle(nx=16, ny=8):
    cfg = cf.Config(nx=nx, ny=ny, nzloc=9, nsubd=3, dt=2e-3).validate()
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-4, 3)
    o.step(2)
    return cfg, o


def _phys(o, cfg):
    out = []
    for q in range(4):
        f = o.state(0)[q].copy()
        out.append(o.horfft(f, 1))
    return np.stack(out)


def parse_unformatted(path, cfg):
    r = records(path)
    assert len(r) == 9
    t = struct.unpack("<d", r[0])[0]
    dims = struct.unpack("<4i", r[1])
    x, y, z = (np.frombuffer(r[k], "<f8") for k in (2, 3, 4))
    shp = (cfg.nz, cfg.ny, cfg.nxpp)
    f = np.stack([np.frombuffer(r[5 + q], "<f4").reshape(shp) for q in range(4)])
    return t, dims, x, y, z, f


def parse_formatted(path, cfg):
    lines = open(path).read().split("\n")
    assert lines[-1] == ""
    lines = lines[:-1]
    for ln in lines:
        if ln is lines[1]:
            continue
        assert len(ln) % 14 == 0 and 14 <= len(ln) <= 70, repr(ln)
    vals = [[float(ln[c:c + 14]) for c in range(0, len(ln), 14)] for k, ln in enumerate(lines) if k != 1]
    dims = [int(lines[1][c:c + 10]) for c in range(0, len(lines[1]), 10)]
    flat = [v for row in vals for v in row]
    return dims, flat, lines


def test_plotf_unformatted(tmp_path):
    cfg, o = _oracle()
    before = o.state(0)
    o.plotf(tmp_path / "p.dat", 0)
    assert np.array_equal(o.state(0), before)
    t, dims, x, y, z, f = parse_unformatted(tmp_path / "p.dat", cfg)
    assert t == o.scalars()[0] and dims == (cfg.nx, cfg.ny, cfg.nz, cfg.ntot)
    xl = 2 * math.pi / (2 * math.pi / cfg.xlen)
    assert np.allclose(x, np.arange(cfg.nx) * xl / cfg.nx, rtol=0, atol=1e-15)
    assert np.array_equal(z, o.tables()["z"]) and len(y) == cfg.ny
    ph = _phys(o, cfg)
    assert np.array_equal(f, ph.astype(np.float32))
    assert not f[..., cfg.nx:].any()


def test_plotf_formatted(tmp_path):
    cfg, o = _oracle(nx=16, ny=4)
    o.plotf(tmp_path / "p.txt", 1)
    dims, flat, lines = parse_formatted(tmp_path / "p.txt", cfg)
    assert dims == [cfg.nx, cfg.ny, cfg.nz, cfg.ntot]
    n_head = 1 + cfg.nx + cfg.ny + cfg.nz
    assert len(flat) == n_head + 4 * cfg.ntot
    ph = _phys(o, cfg).ravel()
    got = np.array(flat[n_head:])
    assert np.all(np.abs(got - ph) <= 5.0001e-6 * np.abs(ph) + 1e-300)  # 6 digits of a 0.dddddd mantissa
    # the fields form one list: only its last line may be short
    field_lines = lines[1 + 1 + math.ceil(cfg.nx / 5) + math.ceil(cfg.ny / 5) + math.ceil(cfg.nz / 5):]
    assert all(len(ln) == 70 for ln in field_lines[:-1])


def test_fortran_e_format_cases(tmp_path):
    """Ew.d with w=14, d=6 as ifort prints it: [-]0.dddddd E[+-]ee."""
    cfg = cf.Config(nx=4, ny=1, nzloc=3, nsubd=1, dt=1.0, xlen=4.0).validate()
    o = Oracle(cfg)
    # x = 0, 1, 2, 3 (xl = 4): the grid line of the formatted file
    o.plotf(tmp_path / "g.txt", 1)
    lines = open(tmp_path / "g.txt").read().split("\n")
    assert lines[2] == "  0.000000E+00  0.100000E+01  0.200000E+01  0.300000E+01"
    assert lines[0] == "  0.000000E+00"
    from oracle import format_e14_6 as f
    cases = {0.9999996: "  0.100000E+01", -2.5: " -0.250000E+01", 1.5e-5: "  0.150000E-04",
             123456.7: "  0.123457E+06", 1e100: "  0.100000+101", -1e-120: " -0.100000-119",
             0.1: "  0.100000E+00", 9.9999949e-3: "  0.999999E-02", 9.9999994e-3: "  0.100000E-01"}
    for v, want in cases.items():
        assert f(v) == want, (v, f(v))


def legendre_spectra(o, cfg, field):
    """speclegencalc (filtering.f:1110-1221) in numpy from the oracle's tables:
    x row at y index nyh (1-based), mean over x of |a_k| per subdomain."""
    tb = o.tables()
    N, ns = cfg.nzloc, cfg.nsubd
    ph = o.horfft(field.copy(), 1)
    row = ph[:, cfg.ny // 2 - 1, :cfg.nx]                  # (nz, nx)
    out = np.zeros((ns, N))
    for ks in range(ns):
        col = row[ks * N:(ks + 1) * N, :]                  # (N, nx)
        s = (tb["alpol"] * tb["wg"][None, :]) @ col        # s[k, i] = sum_j wg_j P_k(z_j) f_j
        fac = np.array([k + 0.5 for k in range(N - 1)] + [0.5 * (N - 1)])
        out[ks] = np.abs(fac[:, None] * s).mean(axis=1)
    return out


def parse_speclegen(path, ns):
    rows = {}
    cur = None
    for ln in open(path).read().split("\n")[:-1]:
        if ln.startswith(" ") and ln[1:3].strip().isdigit() and ln[3:5] == "  ":
            cur = int(ln[1:3])
            rows[cur] = []
            body = ln[5:]
        else:
            body = ln
        rows[cur] += [float(body[c:c + 12]) for c in range(0, len(body), 14)]
    return np.array([rows[k] for k in sorted(rows)]).T        # (ns, N)


def test_oracle_legendre_spectra(tmp_path):
    cfg = cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=2e-3, navgintrfc=0).validate()
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-4, 3)
    o.set_speclegen(2, str(tmp_path))
    o.step(2)
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == sorted("speclegen%s0.004.dat" % c for c in "uvwT")
    for q, c in enumerate("uvwT"):
        got = parse_speclegen(tmp_path / ("speclegen%s0.004.dat" % c), cfg.nsubd)
        ref = legendre_spectra(o, cfg, o.state(0)[q])
        # 6 printed digits; the round-off-level top modes differ by summation order
        assert np.all(np.abs(got - ref) <= 5.0001e-6 * np.abs(ref) + 1e-13 * np.abs(ref).max()), c
        lines = open(tmp_path / ("speclegen%s0.004.dat" % c)).read().split("\n")[:-1]
        assert len(lines) == cfg.nzloc and all(len(ln) == 5 + 12 * 3 + 2 * 2 for ln in lines)


def test_oracle_legendre_spectra_format_reversion_and_names(tmp_path):
    """12 subdomains: 10 values on a kloc's line, the other 2 on the next
    (reversion to 10(e12.6,2x)); t = 10.4 -> F6.3 in the name."""
    cfg = cf.Config(nx=8, ny=4, nzloc=5, nsubd=12, dt=5.2, navgintrfc=0, xnu=1.0, xkappa=1.0).validate()
    o = Oracle(cfg)
    o.init_mode1(1e-3, 0.0, 1)
    o.set_speclegen(2, str(tmp_path))
    o.step(2)
    p = tmp_path / "speclegenu10.400.dat"
    assert p.exists()
    lines = open(p).read().split("\n")[:-1]
    assert len(lines) == 2 * cfg.nzloc
    assert all(len(lines[2 * k]) == 5 + 12 * 10 + 2 * 9 and len(lines[2 * k + 1]) == 12 * 2 + 2 for k in range(cfg.nzloc))
    got = parse_speclegen(p, cfg.nsubd)
    assert got.shape == (cfg.nsubd, cfg.nzloc)
