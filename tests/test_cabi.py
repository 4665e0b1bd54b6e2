"""The C-ABI library loads and exports every entry point include/iw_b200.h
declares (no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "iw_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:int|void|double|char\s*\*|const char\s*\*)\s*\*?\s*(\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_header_lists_the_drop_in_names():
    names = header_functions()
    for n in ("horfft_", "dpdz_", "calcuvwt_", "convec_", "penalty_main_", "bandlu_solve_",
              "filter_3dlegenfourier_", "filter_legenpen_", "interface_avg3d_", "abvar1_", "bdfvarv_",
              "iw_init", "iw_step", "iw_download_state"):
        assert n in names


def test_library_exports_every_declared_symbol():
    import iwrepo_b200 as iw
    if not os.path.exists(iw.LIB_PATH):
        iw.build()
    lib = ctypes.CDLL(iw.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert missing == []
    assert sorted(iw.EXPORTS) == header_functions()


def test_multistep_entry_points_host_only():
    """multistep.f functions are pure host arithmetic in the library."""
    import iwrepo_b200 as iw
    from oracle import multistep as om
    for name in ("abvar1", "abvar2", "abvar3", "bdfvarv", "bdfvar1", "bdfvar2", "bdfvar3"):
        for dts in ((0.1, 0.1, 0.1), (0.1, 0.125, 0.125), (0.08, 0.1, 0.1)):
            assert iw.multistep(name, *dts) == om(name, *dts)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import iwrepo_b200._lib as L
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(L, "_lib", None)
    with pytest.raises(L.IwError):
        L.lib()


def test_dt_rule_entry_point_host_only(golden):
    """iw_dt_rule (maxcalc's adaptive rule, pure host code) replays the
    recorded run's 18 changes and agrees bit for bit with the oracle's rule
    on every branch."""
    import itertools
    import iwrepo_b200 as iw
    import oracle
    from test_oracle_pins import replay_dt_run, wave_omega
    run = golden["dt_run"]
    got = replay_dt_run(iw.dt_rule, run)
    assert len(got) == len(run["changes"])
    for (t, dt), (rt, rdt) in zip(got, run["changes"]):
        assert abs(t - rt) <= 1e-13 * rt and abs(dt - rdt) <= 1e-14 * rdt
    om = wave_omega(2 * 3.141592653589793, 1.0, 1.0)
    for cx, cz, t, dt in itertools.product((0.0, 0.1, 0.16, 0.17), (0.0, 0.05, 0.1, 0.5, 0.7, 0.71, float("nan")),
                                           (0.0, 2.0, 2.1, 2.2, 50.0), (0.1, 0.3, 0.4, 1.0)):
        assert iw.dt_rule(cx, cz, t, dt, om) == oracle.dt_rule(cx, cz, t, dt, om)
