"""Run configuration: dim.h dims, input.dat namelists and subd.dat.

The reference reads its configuration from three places (main.f:185-194,
main.f:261-267, setup.f:316-325):

* ``dim.h`` compile-time PARAMETERs nx, ny, nzloc, nsubd (here: runtime);
* ``input.dat`` namelists ``&inputs``, ``&params``, ``&mflags``;
* ``subd.dat``: the subdomain count, then (z0, h) per subdomain.

This module parses those files, validates them on the host (the reference
validates nothing: FFTFAX prints "INVALID N" and carries on, fft.f:1515), and
fills the ``iw_dims`` / ``iw_params`` C structs of ``include/iw_b200.h``.
It also defines the synthetic workloads of the benchmark suite (C0-C4).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
import re
from typing import Dict, List, Optional, Sequence

IW_MAX_SUBD = 64
IW_MAX_NZLOC = 64
IW_BC_FREESLIP = 0
IW_BC_NOSLIP = 1
IW_PADDLE_OFF, IW_PADDLE_ALL_LEVELS, IW_PADDLE_ABOVE_BOTTOM = 0, 1, 2
IW_PREC_FP64 = 0
IW_PREC_MIXED = 1
IW_SOLVE_AUTO = 0
IW_SOLVE_LU = 1


class ConfigError(ValueError):
    """An invalid dimension, radix, namelist value or subdomain table."""


class IwDims(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nzloc", C.c_int32), ("nsubd", C.c_int32)]


class IwParams(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("xlen", C.c_double), ("ylen", C.c_double), ("zlen", C.c_double),
        ("brunt", C.c_double), ("xnu", C.c_double), ("xkappa", C.c_double),
        ("grav", C.c_double), ("rho0", C.c_double), ("umax", C.c_double),
        ("xacrit", C.c_double), ("xbcrit", C.c_double), ("zcen", C.c_double),
        ("fwave", C.c_double),
        ("amp", C.c_double), ("p", C.c_double), ("pf", C.c_double), ("fackc", C.c_double),
        ("facdir", C.c_double), ("facneumn", C.c_double), ("facrobin", C.c_double),
        ("ispecfilternl", C.c_int32), ("ispecfilterexp", C.c_int32),
        ("nspecfilterexp", C.c_int32), ("navgintrfc", C.c_int32),
        ("bc_variant", C.c_int32), ("meanu_damping", C.c_int32), ("forcing", C.c_int32),
        ("precision", C.c_int32), ("solver", C.c_int32), ("imaxcalc", C.c_int32),
        ("z0", C.c_double * IW_MAX_SUBD), ("zh", C.c_double * IW_MAX_SUBD),
    ]


class IwCoefs(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("fac1", "fac2", "fac3", "bdf1", "bdf2", "bdf3", "bdfv", "dt")]


class IwDiagOut(C.Structure):
    _fields_ = [
        ("ke", C.c_double), ("eps", C.c_double),
        ("umin", C.c_double), ("umax", C.c_double), ("vmin", C.c_double), ("vmax", C.c_double),
        ("wmin", C.c_double), ("wmax", C.c_double), ("tmin", C.c_double), ("tmax", C.c_double),
        ("cflx", C.c_double), ("cfly", C.c_double), ("cflz", C.c_double),
        ("wrms_bottom", C.c_double), ("t", C.c_double), ("dt", C.c_double),
        ("istep", C.c_int32), ("interface_avg_count", C.c_int32 * 4),
    ]


def _radices_ok(n: int) -> bool:
    for r in (2, 3, 5):
        while n % r == 0 and n > 1:
            n //= r
    return n == 1


@dataclasses.dataclass
class Config:
    """dims + namelist values + subdomain table of one run."""

    nx: int
    ny: int
    nzloc: int
    nsubd: int
    dt: float
    xlen: float = 2 * math.pi
    ylen: float = 2 * math.pi
    zlen: float = 1.0
    brunt: float = 1.0
    xnu: float = 1e-3
    xkappa: float = 1e-3
    grav: float = 1.0
    rho0: float = 1.0
    umax: float = 0.01
    xacrit: float = 0.0
    xbcrit: float = 0.84
    zcen: float = 0.13
    fwave: float = 8.0
    amp: float = 36.0
    p: float = 4.0
    pf: float = 4.0
    fackc: float = 0.0
    facdir: float = 1.0
    facneumn: float = 1.0
    facrobin: float = 1.0e4
    ispecfilternl: int = 1
    ispecfilterexp: int = 1
    nspecfilterexp: int = 1
    navgintrfc: int = 1
    bc_variant: int = IW_BC_NOSLIP
    meanu_damping: int = 1
    forcing: int = 0
    precision: int = IW_PREC_FP64
    solver: int = IW_SOLVE_AUTO
    imaxcalc: int = 0
    z0: Optional[List[float]] = None
    zh: Optional[List[float]] = None
    name: str = "custom"

    def __post_init__(self):
        if (self.z0 is None or self.zh is None) and self.nsubd >= 1:
            h = self.zlen / self.nsubd
            self.z0 = [k * h for k in range(self.nsubd)]
            self.zh = [h] * self.nsubd

    # -- derived sizes -------------------------------------------------
    @property
    def nz(self) -> int:
        return self.nzloc * self.nsubd

    @property
    def nxpp(self) -> int:
        return self.nx + 2

    @property
    def ntot(self) -> int:
        return self.nxpp * self.ny * self.nz

    @property
    def ncol(self) -> int:
        return (self.nx // 2 + 1) * self.ny

    @property
    def grid_points(self) -> int:
        return self.nx * self.ny * self.nz

    def validate(self) -> "Config":
        """Host-side checks of what the reference leaves unchecked."""
        if self.nx < 4 or self.nx % 2 or not _radices_ok(self.nx):
            raise ConfigError(f"nx={self.nx}: need an even length with radices 2,3,5 (FFTFAX)")
        if self.ny < 1 or (self.ny > 1 and (self.ny % 2 or not _radices_ok(self.ny))):
            raise ConfigError(f"ny={self.ny}: need 1 or an even length with radices 2,3,5 (CFTFAX)")
        if not 3 <= self.nzloc <= IW_MAX_NZLOC:
            raise ConfigError(f"nzloc={self.nzloc} outside [3,{IW_MAX_NZLOC}]")
        if not 1 <= self.nsubd <= IW_MAX_SUBD:
            raise ConfigError(f"nsubd={self.nsubd} outside [1,{IW_MAX_SUBD}]")
        if self.z0 is None or len(self.z0) != self.nsubd or len(self.zh) != self.nsubd:
            raise ConfigError("subd.dat table length differs from nsubd")
        for ks, (a, h) in enumerate(zip(self.z0, self.zh)):
            if not (h > 0 and math.isfinite(h) and math.isfinite(a)):
                raise ConfigError(f"subdomain {ks + 1}: height {h} must be positive and finite")
            if ks > 0:
                prev_top = self.z0[ks - 1] + self.zh[ks - 1]
                if abs(prev_top - a) > 1e-9 * max(1.0, abs(a)):
                    raise ConfigError(f"subdomain {ks + 1} starts at {a}, previous ends at {prev_top}")
        if abs(self.z0[0]) > 1e-12 or abs(sum(self.zh) - self.zlen) > 1e-9 * max(1.0, self.zlen):
            raise ConfigError(f"subdomains cover [{self.z0[0]}, {self.z0[0] + sum(self.zh)}], zlen={self.zlen}")
        for name in ("dt", "xlen", "ylen", "zlen", "xnu", "xkappa", "grav", "rho0"):
            v = getattr(self, name)
            if not (v > 0 and math.isfinite(v)):
                raise ConfigError(f"{name}={v} must be positive and finite")
        if self.nspecfilterexp < 1:
            raise ConfigError("nspecfilterexp must be >= 1")
        if self.bc_variant not in (IW_BC_FREESLIP, IW_BC_NOSLIP):
            raise ConfigError(f"bc_variant={self.bc_variant}")
        if self.precision not in (IW_PREC_FP64, IW_PREC_MIXED):
            raise ConfigError(f"precision={self.precision}")
        if self.forcing not in (IW_PADDLE_OFF, IW_PADDLE_ALL_LEVELS, IW_PADDLE_ABOVE_BOTTOM):
            raise ConfigError(f"forcing={self.forcing}")
        if self.imaxcalc not in (0, 1):
            raise ConfigError(f"imaxcalc={self.imaxcalc}")
        return self

    # -- C structs -----------------------------------------------------
    def c_dims(self) -> IwDims:
        return IwDims(self.nx, self.ny, self.nzloc, self.nsubd)

    def c_params(self) -> IwParams:
        p = IwParams()
        for f, _ in IwParams._fields_:
            if f in ("z0", "zh"):
                continue
            setattr(p, f, getattr(self, f))
        for k in range(self.nsubd):
            p.z0[k] = self.z0[k]
            p.zh[k] = self.zh[k]
        return p

    def replace(self, **kw) -> "Config":
        return dataclasses.replace(self, **kw)


# ----------------------------------------------------------------------
# input.dat / subd.dat parsing
# ----------------------------------------------------------------------
_NL_GROUP = re.compile(r"[$&](\w+)(.*?)(?:[$&](?:end)?\s*$|/\s*$)", re.S | re.M | re.I)


def parse_namelists(text: str) -> Dict[str, Dict[str, float]]:
    """Parse the ``$inputs ... $`` style namelists of input.dat."""
    groups: Dict[str, Dict[str, float]] = {}
    for m in re.finditer(r"[$&](\w+)(.*?)[$/]", text, re.S):
        name = m.group(1).lower()
        body = m.group(2)
        vals: Dict[str, float] = {}
        for kv in re.finditer(r"(\w+)\s*=\s*([-+0-9.eEdD]+)", body):
            v = kv.group(2).replace("d", "e").replace("D", "e")
            vals[kv.group(1).lower()] = float(v)
        groups[name] = vals
    return groups


def parse_subd(text: str) -> (List[float], List[float]):
    rows = [r.split() for r in text.strip().splitlines() if r.strip()]
    n = int(float(rows[0][0]))
    if len(rows) - 1 < n:
        raise ConfigError(f"subd.dat lists {len(rows) - 1} subdomains, header says {n}")
    z0 = [float(r[0]) for r in rows[1:n + 1]]
    zh = [float(r[1]) for r in rows[1:n + 1]]
    return z0, zh


def from_files(input_dat: str, subd_dat: str, nx: int, ny: int, nzloc: int, nsubd: int,
               **overrides) -> Config:
    """Config of a reference run directory (input.dat + subd.dat + dim.h dims)."""
    nl = parse_namelists(open(input_dat).read())
    z0, zh = parse_subd(open(subd_dat).read())
    if len(z0) < nsubd:
        raise ConfigError(f"subd.dat has {len(z0)} subdomains, dims need {nsubd}")
    i, p, f = nl.get("inputs", {}), nl.get("params", {}), nl.get("mflags", {})
    cfg = Config(
        nx=nx, ny=ny, nzloc=nzloc, nsubd=nsubd, dt=i.get("dtin", 0.1),
        xlen=p["xlen"], ylen=p["ylen"], zlen=p["zlen"], brunt=p["brunt"], xnu=p["xnu"],
        xkappa=p["xkappa"], grav=p["grav"], rho0=p["rho0"], umax=p.get("umax", 0.0),
        xacrit=p.get("xacrit", 0.0), xbcrit=p.get("xbcrit", 0.0), zcen=p.get("zcen", 0.0),
        fwave=i.get("fwave", 0.0), amp=f["amp"], p=f["p"], pf=f["pf"], fackc=f.get("fackc", 0.0),
        facdir=f["facdir"], facneumn=f["facneumn"], facrobin=f["facrobin"],
        ispecfilternl=int(f["ispecfilternl"]), ispecfilterexp=int(f["ispecfilterexp"]),
        nspecfilterexp=int(f["nspecfilterexp"]), navgintrfc=int(f["navgintrfc"]),
        forcing=IW_PADDLE_ALL_LEVELS if p.get("xacrit", 0.0) != 0.0 else IW_PADDLE_OFF, imaxcalc=1,
        z0=z0[:nsubd], zh=zh[:nsubd], name="files")
    cfg = cfg.replace(**overrides)
    return cfg.validate()


# ----------------------------------------------------------------------
# Synthetic workloads (non-dimensional: Lx=Ly=2 pi, H=1, N=1, g=rho0=1,
# nu = 1/Re, kappa = nu (Pr=1), no paddle, no-slip bottom / free-slip top,
# filter order 8 amplitude 36 every step, dt fixed: imaxcalc = 0, so that
# every step does the same work; the reference hard-codes the adaptive step,
# main.f:47, which from_files and shipped_2d keep).
# ----------------------------------------------------------------------
def baseline(name: str, **overrides) -> Config:
    name = name.upper()
    if name == "C0":
        cfg = Config(nx=64, ny=64, nzloc=17, nsubd=4, dt=1e-3, xnu=1e-3, xkappa=1e-3, name="C0")
    elif name == "C2":
        cfg = Config(nx=256, ny=256, nzloc=25, nsubd=8, dt=5e-4, xnu=1 / 2000, xkappa=1 / 2000, name="C2")
    elif name == "C3":
        cfg = Config(nx=512, ny=512, nzloc=33, nsubd=12, dt=2.5e-4, xnu=1 / 5000, xkappa=1 / 5000,
                     name="C3")
    elif name == "C1":
        cfg = Config(nx=256, ny=256, nzloc=25, nsubd=8, dt=1e-3, xnu=1.0, xkappa=1.0, name="C1")
    else:
        raise ConfigError(f"unknown workload {name}")
    return cfg.replace(**overrides).validate()


# initial-condition amplitude and noise of each workload
BASELINE_IC = {"C0": (0.05, 1e-4), "C2": (0.05, 1e-4), "C3": (0.1, 1e-3), "C1": (0.05, 1e-4)}
BASELINE_STEPS = {"C0": 100, "C2": 500, "C3": 1000}


def ensemble_members(n: int = 48, seed: int = 2024) -> List[Config]:
    """Uneven ensemble: Nx=Ny in {64,96,128,192}, 3-8 subdomains of 17-25
    points, Re ~ U[1000,5000] (amplitude and seed drawn alongside)."""
    import random
    rng = random.Random(seed)
    out = []
    for m in range(n):
        nx = rng.choice([64, 96, 128, 192])
        ns = rng.randint(3, 8)
        nzl = rng.randint(17, 25)
        re_ = rng.uniform(1000, 5000)
        cfg = Config(nx=nx, ny=nx, nzloc=nzl, nsubd=ns, dt=5e-4, xnu=1 / re_, xkappa=1 / re_,
                     name=f"E{m}")
        cfg.member_amp = rng.uniform(0.01, 0.1)
        cfg.member_seed = rng.getrandbits(63) | 1
        out.append(cfg.validate())
    return out


def shipped_2d(nx: int = 256, nzloc: int = 25, nsubd: int = 12, **overrides) -> Config:
    """The reference's shipped 2-D forced run (dim.h nx=256, ny=1, 12x25;
    input.dat / subd.dat as shipped), with its values written out.  The
    paddle leaves out the bottom point, as the reference's recorded runs
    do (IW_PADDLE_ABOVE_BOTTOM)."""
    z0 = [0.000, 0.025, 0.075, 0.175, 0.375, 0.775, 1.575, 2.575, 3.375, 3.975, 4.375, 4.775]
    zh = [0.025, 0.050, 0.100, 0.200, 0.400, 0.800, 1.000, 0.800, 0.600, 0.400, 0.400, 0.225]
    cfg = Config(nx=nx, ny=1, nzloc=nzloc, nsubd=nsubd, dt=0.1, xlen=20.0, ylen=1.0, zlen=5.0,
                 brunt=0.2, xnu=1e-5, xkappa=1e-5, grav=9.81, rho0=1e3, umax=0.01, xacrit=2.5,
                 xbcrit=0.84, zcen=0.13, fwave=8.0, amp=35.0, p=5.0, pf=10.0, fackc=0.0,
                 facdir=1.0, facneumn=1.0, facrobin=1e4, ispecfilternl=1, ispecfilterexp=1,
                 nspecfilterexp=1, navgintrfc=1, bc_variant=IW_BC_FREESLIP, meanu_damping=1,
                 forcing=IW_PADDLE_ABOVE_BOTTOM, imaxcalc=1, z0=z0[:nsubd], zh=zh[:nsubd],
                 name="shipped2d")
    return cfg.replace(**overrides).validate()
