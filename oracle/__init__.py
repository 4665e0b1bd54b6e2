"""ORACLE -- test infrastructure only.

ctypes wrapper of ``oracle/liboracle.so``, the CPU FP64 restatement of the
reference time step (see iw_oracle.cpp).  Only the test suite, the smoke test
and the CPU-baseline legs of bench.py use it, always as the checker or the
timed CPU baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from iwrepo_b200.config import Config

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

D = C.c_double
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)


def build() -> str:
    """Compile liboracle.so with oracle/Makefile (no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        for name in ("orc_step", "orc_maxcalc"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_run.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_cache.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_fourier_scale.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_tables.argtypes = [C.c_void_p] + [PD] * 7
        L.orc_set_state.argtypes = [C.c_void_p, C.c_int, PD]
        L.orc_get_state.argtypes = [C.c_void_p, C.c_int, PD]
        L.orc_get_scalars.argtypes = [C.c_void_p, PD]
        L.orc_set_scalars.argtypes = [C.c_void_p, PD]
        L.orc_init_mode1.argtypes = [C.c_void_p, D, D, C.c_uint64]
        L.orc_last_maxcalc.argtypes = [C.c_void_p, PD, PD, PI, PD, PI, PI]
        L.orc_diag.argtypes = [C.c_void_p, PD]
        L.orc_horfft.argtypes = [C.c_void_p, PD, C.c_int, C.c_int]
        L.orc_dpdz.argtypes = [C.c_void_p, PD, PD]
        L.orc_filter3d.argtypes = [C.c_void_p, PD, C.c_int, C.c_int]
        L.orc_filter_legenpen.argtypes = [C.c_void_p, PD, PD]
        L.orc_interface_avg3d.argtypes = [C.c_void_p, PD]
        L.orc_interface_avg3d.restype = C.c_int
        L.orc_penalty_setup.argtypes = [C.c_void_p, D]
        L.orc_penalty_main.argtypes = [C.c_void_p, D, C.c_int, C.c_int, D, D, D, D, PD, PD, PD, PD]
        L.orc_penalty_matrix.argtypes = [C.c_void_p, D, C.c_int, C.c_int, PD]
        L.orc_penalty_params.argtypes = [C.c_void_p, D, C.c_int, C.c_int, PD]
        L.orc_bandlu_solve.argtypes = [C.c_void_p, PD, PD, PD]
        L.orc_bandlu_solve.restype = C.c_int
        L.orc_band_factor.argtypes = [C.c_void_p, PD, PD, PI]
        L.orc_band_factor.restype = C.c_int
        L.orc_get_dt.argtypes = [C.c_void_p, PD]
        L.orc_write_restart.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_plotf.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.orc_plotf.restype = C.c_int
        L.orc_format_e14_6.argtypes = [D, C.c_char_p]
        L.orc_set_animation.argtypes = [C.c_void_p, D, C.c_char_p]
        L.orc_set_speclegen.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
        L.orc_postp.argtypes = [C.c_void_p, PD, PD, D]
        L.orc_animdump_line.argtypes = [D, C.c_int, C.c_int, C.c_char_p, C.c_int]
        L.orc_rhograd.argtypes = [C.c_void_p]
        L.orc_rhograd.restype = D
        L.orc_rhomean.argtypes = [C.c_void_p, D]
        L.orc_rhomean.restype = D
        L.orc_write_restart.restype = C.c_int
        L.orc_read_restart.argtypes = [C.c_void_p, C.c_char_p, C.c_int, D]
        L.orc_read_restart.restype = C.c_int
        L.orc_dt_rule.argtypes = [D, D, D, D, D, PD, PD]
        L.orc_dt_rule.restype = C.c_int
        for n in ("abvar1", "abvar2", "abvar3", "bdfvarv", "bdfvar1", "bdfvar2", "bdfvar3"):
            f = getattr(L, "orc_" + n)
            f.argtypes = [D, D, D]
            f.restype = D
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(PD)


class Oracle:
    """One run of the CPU restatement (state = the reference's COMMON blocks)."""

    def __init__(self, cfg: Config, cache: bool = True, fourier_scale: bool = False):
        self.cfg = cfg
        self._dims = cfg.c_dims()
        self._prm = cfg.c_params()
        self.h = lib().orc_create(C.byref(self._dims), C.byref(self._prm))
        if not self.h:
            raise ValueError(lib().orc_last_error().decode())
        lib().orc_set_cache(self.h, 1 if cache else 0)
        lib().orc_set_fourier_scale(self.h, 1 if fourier_scale else 0)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    # ---- state --------------------------------------------------------
    @property
    def shape(self):
        c = self.cfg
        return (4, c.nz, c.ny, c.nxpp)

    def state(self, level: int = 0) -> np.ndarray:
        a = np.zeros(self.shape)
        lib().orc_get_state(self.h, level, _p(a))
        return a

    def set_state(self, a: np.ndarray, level: int = 0):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.shape)
        lib().orc_set_state(self.h, level, _p(a))

    def scalars(self) -> np.ndarray:
        out = np.zeros(9)
        lib().orc_get_scalars(self.h, _p(out))
        return out

    def set_scalars(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        lib().orc_set_scalars(self.h, _p(s))

    def write_restart(self, path: str):
        """output.f's restart dump (see orc_write_restart)."""
        if lib().orc_write_restart(self.h, str(path).encode()):
            raise RuntimeError(lib().orc_last_error().decode())

    def postp(self, tstart: float = 0.0):
        """postp's TKE budget: the values of an energy.dat and an
        energy_wake.dat line (18 each)."""
        e, w = np.zeros(18), np.zeros(18)
        lib().orc_postp(self.h, _p(e), _p(w), tstart)
        return e, w

    def rhomean(self, z: float) -> float:
        """forcing.f:134-141."""
        return lib().orc_rhomean(self.h, z)

    def rhograd(self) -> float:
        """forcing.f:115-120."""
        return lib().orc_rhograd(self.h)

    def set_speclegen(self, n: int, directory: str = ""):
        """speclegencalc every n steps (see speclegen)."""
        lib().orc_set_speclegen(self.h, n, str(directory).encode())

    def set_animation(self, dtanim: float, directory: str = ""):
        """convec's animation dumps (see anim_dump) every dtanim."""
        lib().orc_set_animation(self.h, dtanim, str(directory).encode())

    def plotf(self, path: str, iform: int = 0):
        """output.f's field dump (see orc_plotf)."""
        if lib().orc_plotf(self.h, str(path).encode(), iform):
            raise RuntimeError(lib().orc_last_error().decode())

    def read_restart(self, path: str, mode: str = "reference", cdtin: float = 1.0):
        """restart.f + main.f:555-632 ("reference": istart = 1 semantics;
        "exact": continue from the file's continuation record)."""
        if lib().orc_read_restart(self.h, str(path).encode(), {"exact": 0, "reference": 1}[mode], cdtin):
            raise RuntimeError(lib().orc_last_error().decode())

    def dt_state(self) -> dict:
        """Current dt and the adaptive step's state (cdt, ivardt, idtstep)."""
        out = np.zeros(4)
        lib().orc_get_dt(self.h, _p(out))
        return dict(dt=out[0], cdt=out[1], ivardt=int(out[2]), idtstep=int(out[3]))

    def tables(self):
        c = self.cfg
        N = c.nzloc
        zp, wg, sg = np.zeros(N), np.zeros(N), np.zeros(N)
        d, d2, al = np.zeros((N, N)), np.zeros((N, N)), np.zeros((N, N))
        z = np.zeros(c.nz)
        lib().orc_tables(self.h, _p(zp), _p(wg), _p(d), _p(d2), _p(al), _p(z), _p(sg))
        return dict(zpts=zp, wg=wg, d=d, d2=d2, alpol=al, z=z, sigma=sg)

    # ---- stepping -----------------------------------------------------
    def init_mode1(self, amplitude: float, noise: float, seed: int):
        lib().orc_init_mode1(self.h, amplitude, noise, seed)

    def step(self, n: int = 1):
        lib().orc_run(self.h, n)

    def last_maxcalc(self):
        probe, mm, cfl = np.zeros(2), np.zeros(8), np.zeros(3)
        mmi, cfli, avg = np.zeros(8, np.int32), np.zeros(9, np.int32), np.zeros(4, np.int32)
        ip = lambda a: a.ctypes.data_as(PI)
        lib().orc_last_maxcalc(self.h, _p(probe), _p(mm), ip(mmi), _p(cfl), ip(cfli), ip(avg))
        return dict(probe=probe, minmax=mm, minmax_idx=mmi, cfl=cfl, cfl_idx=cfli, avg=avg)

    def maxcalc(self):
        lib().orc_maxcalc(self.h)

    def diag(self):
        out = np.zeros(3)
        lib().orc_diag(self.h, _p(out))
        return dict(ke=out[0], eps=out[1], wrms_bottom=out[2])

    # ---- single routines ----------------------------------------------
    def horfft(self, b: np.ndarray, is_: int, nk: int = None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        lib().orc_horfft(self.h, _p(b), is_, nk or self.cfg.nz)
        return b

    def dpdz(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.zeros_like(a)
        lib().orc_dpdz(self.h, _p(a), _p(b))
        return b

    def filter3d(self, f: np.ndarray, ifourier=1, ilegen=1) -> np.ndarray:
        f = np.array(f, dtype=np.float64, order="C")
        lib().orc_filter3d(self.h, _p(f), ifourier, ilegen)
        return f

    def filter_legenpen(self, fin: np.ndarray) -> np.ndarray:
        fin = np.ascontiguousarray(fin, dtype=np.float64)
        out = np.zeros_like(fin)
        lib().orc_filter_legenpen(self.h, _p(fin), _p(out))
        return out

    def interface_avg3d(self, f: np.ndarray):
        f = np.array(f, dtype=np.float64, order="C")
        ic = lib().orc_interface_avg3d(self.h, _p(f))
        return f, ic

    def penalty_setup(self, eps: float):
        lib().orc_penalty_setup(self.h, eps)

    def penalty_main(self, eps, ifbcbot, ifbctop, bcs, rhsr, rhsi):
        rhsr = np.array(rhsr, dtype=np.float64)
        rhsi = np.array(rhsi, dtype=np.float64)
        fr, fi = np.zeros_like(rhsr), np.zeros_like(rhsi)
        lib().orc_penalty_main(self.h, eps, ifbcbot, ifbctop, *bcs, _p(rhsr), _p(rhsi), _p(fr), _p(fi))
        return fr, fi, rhsr, rhsi

    def penalty_matrix(self, eps, ifbcbot, ifbctop) -> np.ndarray:
        nz = self.cfg.nz
        a = np.zeros(nz * nz)
        lib().orc_penalty_matrix(self.h, eps, ifbcbot, ifbctop, _p(a))
        return a.reshape(nz, nz).T.copy()  # row-major A[r, c]

    def penalty_params(self, eps, ifbcbot, ifbctop) -> np.ndarray:
        ns = self.cfg.nsubd
        out = np.zeros(6 * ns)
        lib().orc_penalty_params(self.h, eps, ifbcbot, ifbctop, _p(out))
        return out.reshape(6, ns)

    def band_factor(self, a_rowmajor: np.ndarray):
        nz, N = self.cfg.nz, self.cfg.nzloc
        acm = np.ascontiguousarray(a_rowmajor.T)
        ab = np.zeros((nz, 3 * N + 1))
        ipiv = np.zeros(nz, np.int32)
        info = lib().orc_band_factor(self.h, _p(acm), _p(ab), ipiv.ctypes.data_as(PI))
        return ab, ipiv, info


def multistep(name: str, dt1: float, dt2: float, dt3: float) -> float:
    return getattr(lib(), "orc_" + name)(dt1, dt2, dt3)


def dt_rule(cflx: float, cflz: float, t: float, dt: float, xomega: float):
    """maxcalc's adaptive rule alone: (new dt, cdt) on a change, else None."""
    dn, c = C.c_double(0.0), C.c_double(0.0)
    if lib().orc_dt_rule(cflx, cflz, t, dt, xomega, C.byref(dn), C.byref(c)):
        return dn.value, c.value
    return None


def format_e14_6(v: float) -> str:
    """The oracle's Fortran E14.6 edit descriptor for one value."""
    b = C.create_string_buffer(16)
    lib().orc_format_e14_6(v, b)
    return b.value.decode()


def animdump_line(t: float, n: int, istep: int) -> str:
    """The oracle's animdump.log line (without its newline)."""
    b = C.create_string_buffer(256)
    lib().orc_animdump_line(t, n, istep, b, 256)
    return b.value.decode().rstrip("\n")


def set_threads(n: int):
    lib().orc_set_threads(n)


def max_threads() -> int:
    return lib().orc_max_threads()
