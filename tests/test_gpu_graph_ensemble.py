"""CUDA-graph replay of steps and batched ensembles of uneven runs.

* iw_run(use_graph=1): after the start-up steps every step is one graph
  launch; the state must equal the eager path bit for bit, also after an odd
  number of replayed steps (the history buffers alternate between two
  arrangements) and when eager steps follow.
* iw_ensemble_run: members of different sizes advance together, one graph
  launch per ensemble step; each member must equal the same run done alone.
"""
import numpy as np
import pytest

from iwrepo_b200 import config as cf

pytestmark = pytest.mark.gpu


def _all_levels(s):
    return [s.state(lev) for lev in range(5)]


@pytest.mark.parametrize("precision", [cf.IW_PREC_FP64, cf.IW_PREC_MIXED])
def test_graph_run_equals_eager(precision):
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=32, ny=32, nzloc=9, nsubd=3, dt=1e-3, precision=precision).validate()
    a, b = iw.Solver(cfg), iw.Solver(cfg)
    for s in (a, b):
        s.init_mode1(0.05, 1e-4, 21)
    a.step(10)
    b.run(10, graph=True)  # 3 eager + 7 replayed (odd)
    for x, y in zip(_all_levels(a), _all_levels(b)):
        assert np.array_equal(x, y)
    a.step(3)
    b.step(3)  # eager steps continue from the replayed state
    for x, y in zip(_all_levels(a), _all_levels(b)):
        assert np.array_equal(x, y)
    assert a.diag()["istep"] == b.diag()["istep"] == 13
    a.close()
    b.close()


def test_ensemble_of_uneven_members_equals_individual_runs():
    import iwrepo_b200 as iw
    shapes = [(32, 9, 3), (48, 13, 2), (16, 17, 4)]
    cfgs = [cf.Config(nx=nx, ny=nx, nzloc=nz, nsubd=ns, dt=1e-3, xnu=1 / (1000 + 700 * m), xkappa=1 / (1000 + 700 * m),
                      precision=cf.IW_PREC_MIXED).validate() for m, (nx, nz, ns) in enumerate(shapes)]
    ens = [iw.Solver(c) for c in cfgs]
    alone = [iw.Solver(c) for c in cfgs]
    for m, (e, a) in enumerate(zip(ens, alone)):
        e.init_mode1(0.02 + 0.03 * m, 1e-4, 100 + m)
        a.init_mode1(0.02 + 0.03 * m, 1e-4, 100 + m)
    iw.ensemble_run(ens, 9)
    for a in alone:
        a.step(9)
    for e, a in zip(ens, alone):
        for x, y in zip(_all_levels(e), _all_levels(a)):
            assert np.array_equal(x, y)
    for s in ens + alone:
        s.close()


@pytest.mark.parametrize("precision,tol", [(cf.IW_PREC_FP64, 1e-11), (cf.IW_PREC_MIXED, 1e-5)])
def test_autotune_keeps_results(precision, tol):
    """iw_autotune only changes launch choices: the state is untouched and the
    following steps agree with an untuned run to rounding."""
    import iwrepo_b200 as iw
    cfg = cf.Config(nx=32, ny=32, nzloc=9, nsubd=3, dt=1e-3, precision=precision).validate()
    a, b = iw.Solver(cfg), iw.Solver(cfg)
    for s in (a, b):
        s.init_mode1(0.05, 1e-4, 31)
    a.step(2)
    b.step(2)
    before = b.state(0)
    ch = b.autotune()
    assert ch["y_tile"] in (2, 4, 8) and ch["stage_a"] in ("register", "tiled")
    assert ch["stage_e"] in ("register", "tiled", "tiled-bulk", "tiled-bulk-constant-operators")
    assert ch["x_row_threads"] in (128, 256)
    assert np.array_equal(before, b.state(0))
    a.step(6)
    b.step(6)
    for x, y in zip(_all_levels(a), _all_levels(b)):
        for q in range(4):
            assert np.linalg.norm(x[q] - y[q]) <= tol * max(np.linalg.norm(y[q]), 1e-300)
    a.close()
    b.close()
