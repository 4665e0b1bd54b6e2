"""Loader of libiwb200.so (the CUDA library behind include/iw_b200.h).

The product path has no CPU fallback: if the shared library is missing or no
CUDA device is present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from .config import IwDims, IwParams, IwCoefs, IwDiagOut

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libiwb200.so")
CSRC = os.path.join(HERE, "csrc")

_lib = None

PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)

# every entry point declared in include/iw_b200.h
EXPORTS = [
    "iw_init", "iw_destroy", "iw_last_error", "iw_last_status", "iw_upload_state", "iw_download_state", "iw_init_mode1",
    "iw_write_restart", "iw_read_restart", "iw_write_fields", "iw_wait_fields", "iw_set_animation", "iw_set_speclegen", "iw_postp", "iw_set_postp", "iw_step", "iw_run", "iw_ensemble_run", "iw_autotune", "iw_set_launch", "iw_get_launch", "iw_step_coefs", "iw_set_coefs", "iw_diag", "iw_sync", "iw_field_ptr", "iw_stream",
    "iw_device_bytes", "iw_helm_solve_batched", "iw_bind", "iw_profile", "iw_profile_read", "iw_mean_profiles",
    "horfft_", "dpdz_", "filter_3dlegenfourier_", "filter_legenpen_", "interface_avg3d_",
    "penalty_main_", "bandlu_solve_", "iw_bandlu_solve_noalloc", "penalty_setup_", "convec_", "calcuvwt_",
    "abvar1_", "abvar2_", "abvar3_", "bdfvarv_", "bdfvar1_", "bdfvar2_", "bdfvar3_", "iw_dt_rule",
]


class IwError(RuntimeError):
    """A nonzero status of the C ABI; .code holds the IW_ERR_* value."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


def build(verbose: bool = False) -> str:
    """Compile libiwb200.so for sm_100a (nvcc cross-compiles without a GPU)."""
    r = subprocess.run(["make", "-s", "-C", CSRC], capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise IwError("building libiwb200.so failed:\n" + (r.stdout or "") + (r.stderr or ""))
    return LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise IwError(f"{LIB_PATH} is not built; run iwrepo_b200.build() (there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.iw_init.argtypes = [C.POINTER(IwDims), C.POINTER(IwParams), C.c_int, C.POINTER(vp)]
    L.iw_destroy.argtypes = [vp]
    L.iw_last_status.restype = C.c_int
    L.iw_last_error.restype = C.c_char_p
    L.iw_upload_state.argtypes = [vp, PD, PD, PD, PD, PD, C.c_double, C.c_int]
    L.iw_download_state.argtypes = [vp, PD, PD, PD, PD, PD]
    L.iw_init_mode1.argtypes = [vp, C.c_double, C.c_double, C.c_uint64]
    L.iw_step.argtypes = [vp]
    L.iw_run.argtypes = [vp, C.c_int, C.c_int]
    L.iw_ensemble_run.argtypes = [C.POINTER(vp), C.c_int, C.c_int]
    L.iw_autotune.argtypes = [vp, PI]
    L.iw_set_launch.argtypes = [vp, C.c_int, C.c_int]
    L.iw_get_launch.argtypes = [vp, C.c_int, PI]
    L.iw_step_coefs.argtypes = [vp, C.POINTER(IwCoefs)]
    L.iw_set_coefs.argtypes = [vp, C.POINTER(IwCoefs), C.c_double]
    L.iw_diag.argtypes = [vp, C.POINTER(IwDiagOut)]
    L.iw_sync.argtypes = [vp]
    L.iw_field_ptr.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.iw_stream.argtypes = [vp, C.POINTER(vp)]
    L.iw_device_bytes.argtypes = [vp, C.POINTER(C.c_size_t)]
    L.iw_helm_solve_batched.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp, vp, C.c_int]
    L.iw_bandlu_solve_noalloc.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp]
    L.iw_bind.argtypes = [vp]
    L.iw_profile.argtypes = [vp, C.c_int]
    L.iw_mean_profiles.argtypes = [vp, PD]
    L.iw_profile_read.argtypes = [vp, PD, C.POINTER(C.c_long)]
    L.horfft_.argtypes = [PD, PI, PI]
    L.horfft_.restype = None
    L.dpdz_.argtypes = [PD, PD]
    L.dpdz_.restype = None
    L.filter_3dlegenfourier_.argtypes = [PD, PI, PI, PI]
    L.filter_3dlegenfourier_.restype = None
    L.filter_legenpen_.argtypes = [PD, PD, PD, PI, PI]
    L.filter_legenpen_.restype = None
    L.interface_avg3d_.argtypes = [PD, PI]
    L.interface_avg3d_.restype = None
    L.penalty_main_.argtypes = [PD, PI, PD, PD, PD, PD, PI, PI, PD, PD, PD, PD]
    L.penalty_main_.restype = None
    L.bandlu_solve_.argtypes = [PD, PD, PD, PI]
    L.bandlu_solve_.restype = None
    L.penalty_setup_.argtypes = [PD]
    L.penalty_setup_.restype = None
    L.convec_.argtypes = [PI, PI, PI]
    L.convec_.restype = None
    L.calcuvwt_.argtypes = [PI, PI, PI, PI]
    L.calcuvwt_.restype = None
    for n in ("abvar1_", "abvar2_", "abvar3_", "bdfvarv_", "bdfvar1_", "bdfvar2_", "bdfvar3_"):
        getattr(L, n).argtypes = [PD, PD, PD]
        getattr(L, n).restype = C.c_double
    L.iw_write_restart.argtypes = [vp, C.c_char_p]
    L.iw_write_fields.argtypes = [vp, C.c_char_p, C.c_int]
    L.iw_wait_fields.argtypes = [vp]
    L.iw_set_animation.argtypes = [vp, C.c_double, C.c_char_p]
    L.iw_set_speclegen.argtypes = [vp, C.c_int, C.c_char_p]
    L.iw_postp.argtypes = [vp, PD, PD]
    L.iw_set_postp.argtypes = [vp, C.c_int, C.c_double, C.c_char_p]
    L.iw_read_restart.argtypes = [vp, C.c_char_p, C.c_int, C.c_double]
    L.iw_dt_rule.argtypes = [C.c_double] * 5 + [PD, PD]
    L.iw_dt_rule.restype = C.c_int
    _lib = L
    return L


def check(rc: int):
    if rc != 0:
        raise IwError(f"iw error {rc}: {lib().iw_last_error().decode()}", rc)
