"""C2 (256^2 x (8x25), FP64) against the oracle at C2's own size over its
full 500 steps, compared with the fingerprint the oracle left in
tests/golden/c2_fingerprint.json (made by tests/golden/make_c2_fingerprint.py,
about 4 h on 6 host threads; the full state, 420 MB, is too large to commit).

* KE and dissipation every 10 steps: 1e-10 relative.
* Per field: the L2 norm (1e-10 relative), the inner product with a seeded
  random field (1e-10 of norm times the random field's norm, Cauchy-Schwarz
  for a 1e-10 relative L2 difference) and 16 probe values (1e-8 of the field's
  rms: pointwise differences may exceed the rms difference).
"""
import importlib.util
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _generator():
    spec = importlib.util.spec_from_file_location("make_c2_fingerprint",
                                                  os.path.join(HERE, "golden", "make_c2_fingerprint.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_c2_matches_oracle_fingerprint():
    import iwrepo_b200 as iw
    from iwrepo_b200 import config as cf
    fp = json.load(open(os.path.join(HERE, "golden", "c2_fingerprint.json")))
    assert fp["steps"] == 500 and len(fp["series"]) == 50
    gen = _generator()
    cfg = cf.baseline("C2")
    s = iw.Solver(cfg)
    s.init_mode1(fp["amp"], fp["noise"], fp["seed"])
    for rec in fp["series"]:
        s.step(10)
        d = s.diag()
        assert abs(d["ke"] - rec["ke"]) <= 1e-10 * abs(rec["ke"]), rec["step"]
        assert abs(d["eps"] - rec["eps"]) <= 1e-10 * abs(rec["eps"]), rec["step"]
    st = s.state(0)
    got = gen.fingerprint(st)
    n = st[0].size
    rnorm = np.sqrt(n)  # norm of the standard-normal field, to within a few 1e-3
    for name, ref in fp["fields"].items():
        g = got[name]
        assert abs(g["norm"] - ref["norm"]) <= 1e-10 * ref["norm"], name
        assert abs(g["dot"] - ref["dot"]) <= 1.1e-10 * ref["norm"] * rnorm, name
        rms = ref["norm"] / np.sqrt(n)
        assert np.all(np.abs(np.array(g["probes"]) - np.array(ref["probes"])) <= 1e-8 * rms), name
    s.close()
