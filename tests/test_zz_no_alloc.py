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


@pytest.mark.parametrize("nzloc,nsubd,nrhs", [(9, 3, 1), (25, 8, 2), (25, 8, 1), (25, 64, 2)])
def test_bandlu_noalloc_at_c1_size_and_at_its_limit(nzloc, nsubd, nrhs):
    """C1's 8 x 25 system, one and two right-hand sides, and the largest
    system the scratch takes (nzloc = 25, nsubd = 64: nz = 1600, band
    (3*25+1)*1600 = 121,600 of 131,072 doubles): bit-equal to bandlu_solve_
    on two consecutive calls, normwise backward error below 1e-14 (the
    penalty rows reach 3e6 at these sizes, so the residual itself is not
    small relative to the right-hand side)."""
    import torch
    import iwrepo_b200 as iw
    from iwrepo_b200 import _lib
    from oracle import Oracle

    cfg = cf.Config(nx=4, ny=2, nzloc=nzloc, nsubd=nsubd, dt=1e-3).validate()
    n = cfg.nz
    s, o = iw.Solver(cfg), Oracle(cfg)
    L = _lib.lib()
    rng = np.random.default_rng(nzloc * 100 + nsubd)
    for eps, bot, top in [(2e-4, 0, 1), (0.3, 1, 1)]:
        A = o.penalty_matrix(eps, bot, top)
        x1, x2 = rng.standard_normal(n), rng.standard_normal(n)
        ref_r, ref_i = s.bandlu_solve(A, x1, x2)
        a_dev = torch.from_numpy(np.ascontiguousarray(A.T).ravel()).cuda()
        x_dev = torch.from_numpy(np.concatenate([x1, x2][:nrhs])).cuda()
        torch.cuda.synchronize()
        rc = L.iw_bandlu_solve_noalloc(_ptr(a_dev), _ptr(x_dev), nzloc, nsubd, nrhs, None)
        assert rc == 0, L.iw_last_error()
        torch.cuda.synchronize()
        got = x_dev.cpu().numpy()
        assert np.array_equal(got[:n], ref_r)
        if nrhs == 2:
            assert np.array_equal(got[n:], ref_i)
        r = A @ got[:n] - x1
        assert np.max(np.abs(r)) / (np.linalg.norm(A, np.inf) * np.max(np.abs(got[:n]))) < 1e-14
    s.close()


def test_bandlu_noalloc_refuses_systems_beyond_its_scratch():
    import torch
    from iwrepo_b200 import _lib

    L = _lib.lib()
    a_dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    x_dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    # band (3*64+1)*64*64 and (3*26+1)*26*64 exceed 131,072: refused before anything is launched
    for nzloc, nsubd in ((64, 64), (26, 64)):
        rc = L.iw_bandlu_solve_noalloc(_ptr(a_dev), _ptr(x_dev), nzloc, nsubd, 2, None)
        assert rc == IW_ERR_CONFIG
        assert b"fixed scratch" in L.iw_last_error()
    rc = L.iw_bandlu_solve_noalloc(_ptr(a_dev), _ptr(x_dev), 9, 3, 3, None)
    assert rc == IW_ERR_CONFIG
