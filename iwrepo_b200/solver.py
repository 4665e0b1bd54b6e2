"""Host-side mirror of the reference's time-step interface on the B200 library.

``Solver`` owns one device-resident run (the reference's COMMON blocks) and
exposes the reference's subroutines with their names and semantics:

=====================  ==========================================  =========================
method                 reference routine                           device work
=====================  ==========================================  =========================
``step``               main.f:653-1066 (maxcalc, convec,           the fused step kernels
                       calcuvwt, interface_avg3d)
``convec``             solver.f:6-514                              K_A..K_E
``calcuvwt``           calcuvwt_noslip.f / calcuvwt.f              pressure + viscous solves
``horfft``             horfft.f:2-69                               x/y FFT kernels
``dpdz``               derv.f:212-275                              z-derivative kernel
``filter_3dlegenfourier``  filtering.f:811-983                     filter kernel
``interface_avg3d``    penalty.f:714-775                           interface kernels
``penalty_main``       penalty.f:162-251 (+ band_lu.f)             device assembly, LU, solve
``bandlu_solve``       band_lu.f:15-54                             device LU and solve
=====================  ==========================================  =========================

Arrays use the reference layout ``(4 fields, nz, ny, nxpp)`` float64.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .config import Config, IwCoefs, IwDiagOut


def _pd(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ri(v: int):
    return C.byref(C.c_int(int(v)))


def _rd(v: float):
    return C.byref(C.c_double(float(v)))


class Solver:
    """One run on one GPU (fields stay on the device between calls)."""

    def __init__(self, cfg: Config, device: int = 0):
        cfg.validate()
        self.cfg = cfg
        self._dims = cfg.c_dims()
        self._prm = cfg.c_params()
        h = C.c_void_p()
        _lib.check(_lib.lib().iw_init(C.byref(self._dims), C.byref(self._prm), device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().iw_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------
    @property
    def shape(self):
        c = self.cfg
        return (4, c.nz, c.ny, c.nxpp)

    def init_mode1(self, amplitude: float, noise: float, seed: int):
        _lib.check(_lib.lib().iw_init_mode1(self.h, amplitude, noise, seed))

    def set_state(self, uvwt, uvwt_n=None, uvwt_nm=None, s_n=None, s_nm=None, t=0.0, istep=0):
        arrs = []
        for a in (uvwt, uvwt_n, uvwt_nm, s_n, s_nm):
            arrs.append(None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.shape))
        ptrs = [None if a is None else _pd(a) for a in arrs]
        _lib.check(_lib.lib().iw_upload_state(self.h, *ptrs, t, istep))

    def state(self, level: int = 0, out: np.ndarray = None) -> np.ndarray:
        """Download one time level (0: n, 1: n-1, 2: n-2, 3/4: NL terms at
        n-1/n-2) as FP64, into `out` when given (C-contiguous float64 of
        self.shape, e.g. pinned host memory)."""
        if out is None:
            out = np.zeros(self.shape)
        elif out.dtype != np.float64 or out.shape != self.shape or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be C-contiguous float64 of shape %s" % (self.shape,))
        ptrs = [None] * 5
        ptrs[level] = _pd(out)
        _lib.check(_lib.lib().iw_download_state(self.h, *ptrs))
        return out

    def step(self, n: int = 1):
        _lib.check(_lib.lib().iw_run(self.h, n, 0))

    def write_restart(self, path: str):
        """output.f's restart dump through iw_write_restart (the reference's 49
        records plus the continuation record)."""
        _lib.check(_lib.lib().iw_write_restart(self.h, str(path).encode()))

    def write_fields(self, path: str, iform: int = 0, wait: bool = True):
        """plotf's field dump through iw_write_fields (iform 0 unformatted
        REAL*4, 1 formatted 5e14.6).  With wait=False the file is written by a
        host thread while later steps run; call wait_fields() before reading it."""
        _lib.check(_lib.lib().iw_write_fields(self.h, str(path).encode(), iform))
        if wait:
            self.wait_fields()

    def wait_fields(self):
        _lib.check(_lib.lib().iw_wait_fields(self.h))

    def postp(self):
        """postp's TKE budget of the current state (iw_postp): the values of one
        energy.dat line and one energy_wake.dat line (18 each)."""
        e, w = np.zeros(18), np.zeros(18)
        _lib.check(_lib.lib().iw_postp(self.h, _pd(e), _pd(w)))
        return e, w

    def set_postp(self, npostp: int, tstart: float = 0.0, directory: str = ""):
        """Append the budget lines to energy.dat, energy_wake.dat and
        wakescale.dat in directory every npostp steps; <= 0 turns it off."""
        _lib.check(_lib.lib().iw_set_postp(self.h, npostp, tstart, str(directory).encode()))

    def set_speclegen(self, ncalclegspec: int, directory: str = ""):
        """speclegencalc's Legendre spectra of u, v, w, T every ncalclegspec
        steps (speclegen<c><t>.dat in directory); <= 0 turns them off."""
        _lib.check(_lib.lib().iw_set_speclegen(self.h, ncalclegspec, str(directory).encode()))

    def set_animation(self, dtanim: float, directory: str = ""):
        """convec's animation dumps (vortanimout_NNNNN.dat in directory) every
        dtanim of simulated time; dtanim <= 0 turns them off."""
        _lib.check(_lib.lib().iw_set_animation(self.h, dtanim, str(directory).encode()))

    def read_restart(self, path: str, mode: str = "reference", cdtin: float = 1.0):
        """restart.f through iw_read_restart: mode "reference" gives main.f's
        istart = 1 start (cdtin = old dt / new dt), "exact" continues a run
        written by write_restart bit for bit."""
        m = {"exact": 0, "reference": 1}[mode]
        _lib.check(_lib.lib().iw_read_restart(self.h, str(path).encode(), m, cdtin))

    def autotune(self) -> dict:
        """Time this step's launch candidates and keep the fastest (y-tile
        width, stage A / stage E variant, solve variant); the state is not
        changed."""
        ch = (C.c_int * 4)()
        _lib.check(_lib.lib().iw_autotune(self.h, ch))
        names = {3: "tiled-bulk-constant-operators", 2: "tiled-bulk", 1: "register", 0: "tiled", -1: "n/a"}
        solve = {0: "per-task", 1: "system-grouped", 2: "system-grouped-tensor-core",
                 3: "system-grouped-two-rows"}
        out = {"y_tile": ch[0], "stage_a": names[ch[1]], "stage_e": names[ch[2]], "solve": solve[ch[3]]}
        out["solve_roles"] = {role: solve.get(self.get_launch("solve_" + role), "n/a")
                              for role in ("uv", "w", "rho", "pressure")}
        out["x_row_threads"] = self.get_launch("x_row_threads")
        return out

    LAUNCH = {"y_tile": 0, "stage_a": 1, "stage_e": 2, "solve": 3, "solve_uv": 4, "solve_w": 5, "solve_rho": 6,
              "solve_pressure": 7, "x_row_threads": 8}

    def set_launch(self, which: str, value: int):
        """Set one launch choice directly (iw_set_launch)."""
        _lib.check(_lib.lib().iw_set_launch(self.h, self.LAUNCH[which], int(value)))

    def get_launch(self, which: str) -> int:
        """Read one launch choice (iw_get_launch)."""
        v = C.c_int(0)
        _lib.check(_lib.lib().iw_get_launch(self.h, self.LAUNCH[which], C.byref(v)))
        return v.value

    def run(self, n: int, graph: bool = True):
        """n steps; with graph=True the invariant steady-state step is replayed
        from captured CUDA graphs (identical results, one launch per step)."""
        _lib.check(_lib.lib().iw_run(self.h, n, 1 if graph else 0))

    def step_coefs(self, fac, bdf, bdfv, dt):
        c = IwCoefs(fac[0], fac[1], fac[2], bdf[0], bdf[1], bdf[2], bdfv, dt)
        _lib.check(_lib.lib().iw_step_coefs(self.h, C.byref(c)))

    def set_coefs(self, fac, bdf, bdfv, dt, t):
        """COMMON /ab/ /bdf/ values, dt and t for convec_/calcuvwt_ (iw_set_coefs)."""
        c = IwCoefs(fac[0], fac[1], fac[2], bdf[0], bdf[1], bdf[2], bdfv, dt)
        _lib.check(_lib.lib().iw_set_coefs(self.h, C.byref(c), t))

    def sync(self):
        _lib.check(_lib.lib().iw_sync(self.h))

    def diag(self) -> dict:
        d = IwDiagOut()
        _lib.check(_lib.lib().iw_diag(self.h, C.byref(d)))
        return dict(ke=d.ke, eps=d.eps, t=d.t, dt=d.dt, istep=d.istep, avg=list(d.interface_avg_count),
                    wrms_bottom=d.wrms_bottom, cfl=(d.cflx, d.cfly, d.cflz),
                    minmax=(d.umin, d.umax, d.vmin, d.vmax, d.wmin, d.wmax, d.tmin, d.tmax))

    def mean_profiles(self, out: np.ndarray = None) -> np.ndarray:
        """(4, nz) mean profiles of u, v, w, rho (device -> host, synchronous)."""
        if out is None:
            out = np.zeros(4 * self.cfg.nz)
        _lib.check(_lib.lib().iw_mean_profiles(self.h, _pd(out)))
        return out.reshape(4, self.cfg.nz)

    def device_bytes(self) -> int:
        b = C.c_size_t()
        _lib.check(_lib.lib().iw_device_bytes(self.h, C.byref(b)))
        return b.value

    def field_ptr(self, f: int) -> int:
        p = C.c_void_p()
        _lib.check(_lib.lib().iw_field_ptr(self.h, f, C.byref(p)))
        return p.value

    def stream(self) -> int:
        p = C.c_void_p()
        _lib.check(_lib.lib().iw_stream(self.h, C.byref(p)))
        return p.value

    def profile(self, enable: bool = True):
        _lib.check(_lib.lib().iw_profile(self.h, 1 if enable else 0))

    PHASES = ["stageA", "y_inverse", "x_row_nl", "y_forward", "wall_bc", "stageE", "pressure", "solve_uv",
              "solve_w", "solve_rho", "interface_avg"]

    def profile_read(self) -> dict:
        ms = (C.c_double * 16)()
        n = (C.c_long * 16)()
        _lib.check(_lib.lib().iw_profile_read(self.h, ms, n))
        return {p: (ms[i], n[i]) for i, p in enumerate(self.PHASES)}

    # ------------------------------------------------------------------
    # the reference's subroutines (Fortran-style entry points)
    def _bind(self):
        _lib.lib().iw_bind(self.h)

    def horfft(self, b: np.ndarray, is_: int, nk: int = None) -> np.ndarray:
        self._bind()
        b = np.array(b, dtype=np.float64, order="C")
        _lib.lib().horfft_(_pd(b), _ri(is_), _ri(nk or self.cfg.nz))
        return b

    def dpdz(self, a: np.ndarray) -> np.ndarray:
        self._bind()
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.zeros_like(a)
        _lib.lib().dpdz_(_pd(a), _pd(b))
        return b

    def filter_3dlegenfourier(self, f: np.ndarray, ifourier=1, ilegen=1) -> np.ndarray:
        self._bind()
        f = np.array(f, dtype=np.float64, order="C")
        _lib.lib().filter_3dlegenfourier_(_pd(f), _ri(ifourier), _ri(ilegen), _ri(0))
        return f

    def filter_legenpen(self, fin: np.ndarray) -> np.ndarray:
        self._bind()
        fin = np.ascontiguousarray(fin, dtype=np.float64)
        out = np.zeros_like(fin)
        _lib.lib().filter_legenpen_(_pd(fin), _pd(out), _rd(1.0), _ri(0), _ri(1))
        return out

    def interface_avg3d(self, f: np.ndarray):
        self._bind()
        f = np.array(f, dtype=np.float64, order="C")
        ic = C.c_int(0)
        _lib.lib().interface_avg3d_(_pd(f), C.byref(ic))
        return f, ic.value

    def penalty_setup(self, eps: float):
        self._bind()
        _lib.lib().penalty_setup_(_rd(eps))

    def penalty_main(self, eps, ifbcbot, ifbctop, bcs, rhsr, rhsi):
        """penalty.f:162-251; rhsr/rhsi are scaled by -eps in place (returned)."""
        self._bind()
        rhsr = np.array(rhsr, dtype=np.float64)
        rhsi = np.array(rhsi, dtype=np.float64)
        fr, fi = np.zeros_like(rhsr), np.zeros_like(rhsi)
        L = _lib.lib()
        L.penalty_main_(_rd(eps), _ri(0), _rd(bcs[0]), _rd(bcs[1]), _rd(bcs[2]), _rd(bcs[3]), _ri(ifbcbot),
                        _ri(ifbctop), _pd(rhsr), _pd(rhsi), _pd(fr), _pd(fi))
        return fr, fi, rhsr, rhsi

    def bandlu_solve(self, a_rowmajor: np.ndarray, xr, xi):
        self._bind()
        acm = np.ascontiguousarray(np.asarray(a_rowmajor, dtype=np.float64).T)
        xr = np.array(xr, dtype=np.float64)
        xi = np.array(xi, dtype=np.float64)
        _lib.lib().bandlu_solve_(_pd(acm), _pd(xr), _pd(xi), _ri(0))
        return xr, xi

    def convec(self, istep: int):
        self._bind()
        _lib.lib().convec_(_ri(istep), _ri(0), _ri(self.cfg.ispecfilternl))

    def calcuvwt(self, cpenspecfilter: bool = True):
        self._bind()
        _lib.lib().calcuvwt_(_ri(0), _ri(0), _ri(0), _ri(1 if cpenspecfilter else 0))


def ensemble_run(members, n: int):
    """Advance independent runs of any sizes (Solver objects on one device) by
    n steps each; once all are in steady state, each ensemble step is one
    CUDA-graph launch.  Results equal running each member alone."""
    arr = (C.c_void_p * len(members))(*[m.h for m in members])
    _lib.check(_lib.lib().iw_ensemble_run(arr, len(members), n))


def multistep(name: str, dt1: float, dt2: float, dt3: float) -> float:
    """multistep.f:7-89 through the C ABI (abvar1_ ... bdfvar3_)."""
    return getattr(_lib.lib(), name + "_")(_rd(dt1), _rd(dt2), _rd(dt3))


def dt_rule(cflx: float, cflz: float, t: float, dt: float, xomega: float):
    """maxcalc's adaptive time-step rule (various.f:892-982) through the C ABI
    (iw_dt_rule): (new dt, cdt) when the step changes, else None."""
    dn, c = C.c_double(0.0), C.c_double(0.0)
    if _lib.lib().iw_dt_rule(cflx, cflz, t, dt, xomega, C.byref(dn), C.byref(c)):
        return dn.value, c.value
    return None


def helm_solve_batched(solver: Solver, lam_dev_ptr: int, ncol: int, ifbcbot: int, ifbctop: int, rhs_dev_ptr: int,
                       sol_dev_ptr: int, mode: int = 0):
    """Batched isolated penalty solves on device buffers (see iw_helm_solve_batched)."""
    _lib.check(_lib.lib().iw_helm_solve_batched(solver.h, C.c_void_p(lam_dev_ptr), ncol, ifbcbot, ifbctop,
                                                C.c_void_p(rhs_dev_ptr), C.c_void_p(sol_dev_ptr), mode))
