"""iw_bandlu_solve_noalloc: the banded penalty solve for callers that cannot
allocate device memory while they run (their device memory belongs to a pool
sized at start-up, or a cudaFree would stall their loop).  It must give what
bandlu_solve_ gives, call after call, while reusing one fixed scratch array.

This file is named so that pytest collects it after every other test file.
"""
import ctypes

import numpy as np
import pytest

from iwrepo_b200 import config as cf

pytestmark = pytest.mark.gpu

IW_ERR_CONFIG = 1


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_bandlu_noalloc_matches_bandlu_solve_on_consecutive_calls():
    import torch
    import iwrepo_b200 as iw
    from iwrepo_b200 import _lib
    from oracle import Oracle

    cfg = cf.Config(nx=16, ny=8, nzloc=9, nsubd=3, dt=1e-3).validate()
    n = cfg.nz
    s, o = iw.Solver(cfg), Oracle(cfg)
    L = _lib.lib()
    rng = np.random.default_rng(17)
    # two different systems in a row: the second call must not see anything the
    # first one left in the shared scratch
    for eps, bot, top in [(3e-3, 0, 1), (0.7, 1, 1)]:
        A = o.penalty_matrix(eps, bot, top)  # row major
        x1, x2 = rng.standard_normal(n), rng.standard_normal(n)
        ref_r, ref_i = s.bandlu_solve(A, x1, x2)  # existing entry point, host arrays
        a_dev = torch.from_numpy(np.ascontiguousarray(A.T).ravel()).cuda()  # column major
        x_dev = torch.from_numpy(np.concatenate([x1, x2])).cuda()
        torch.cuda.synchronize()
        rc = L.iw_bandlu_solve_noalloc(_ptr(a_dev), _ptr(x_dev), cfg.nzloc, cfg.nsubd, 2, None)
        assert rc == 0, L.iw_last_error()
        torch.cuda.synchronize()
        got = x_dev.cpu().numpy()
        # same packing, factorisation and solve kernels as bandlu_solve_: identical bits
        assert np.array_equal(got[:n], ref_r) and np.array_equal(got[n:], ref_i)
        assert np.linalg.norm(A @ got[:n] - x1) / np.linalg.norm(x1) < 1e-12


def test_bandlu_noalloc_refuses_systems_beyond_its_scratch():
    import torch
    from iwrepo_b200 import _lib

    L = _lib.lib()
    a_dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    x_dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    # nz = 64*64 = 4096 > 3072: refused before anything is launched
    rc = L.iw_bandlu_solve_noalloc(_ptr(a_dev), _ptr(x_dev), 64, 64, 2, None)
    assert rc == IW_ERR_CONFIG
    assert b"fixed scratch" in L.iw_last_error()
    rc = L.iw_bandlu_solve_noalloc(_ptr(a_dev), _ptr(x_dev), 9, 3, 3, None)
    assert rc == IW_ERR_CONFIG
