"""B200-native time step of the jmsegret/IWrepo stratified Boussinesq solver.

Fourier pseudo-spectral in x and y, Legendre multidomain penalty in z,
exponential filtering and the stiffly stable / BDF3 scheme with a pressure
projection, run as hand-written sm_100a kernels on device-resident fields.
The C ABI is include/iw_b200.h; this package is the Python host side.
"""
from .config import (Config, ConfigError, baseline, ensemble_members, from_files, shipped_2d,
                     IW_BC_FREESLIP, IW_BC_NOSLIP, IW_PREC_FP64, IW_PREC_MIXED)
from ._lib import build, IwError, LIB_PATH, EXPORTS
from .solver import Solver, ensemble_run, multistep, dt_rule, helm_solve_batched

__all__ = ["Config", "ConfigError", "baseline", "ensemble_members", "from_files", "shipped_2d", "build",
           "IwError", "Solver", "ensemble_run", "multistep", "dt_rule", "helm_solve_batched", "IW_BC_FREESLIP", "IW_BC_NOSLIP",
           "IW_PREC_FP64", "IW_PREC_MIXED", "LIB_PATH", "EXPORTS"]
