"""Fingerprint of C2 after its 500 FP64 steps of the oracle, for the GPU parity
test at C2's size (256^2 x (8x25)), where the full state (420 MB) is too large
to commit.

Run on any CPU (about 3 hours on 8 threads):
    python tests/golden/make_c2_fingerprint.py [steps] [threads] [output]
(defaults: 500 steps, all threads, tests/golden/c2_fingerprint.json).
Writes:
* per field (u, v, w, rho): the L2 norm, the inner product with a seeded
  random field (numpy default_rng(7), standard normal, same shape) and 16
  probe values at fixed indices;
* KE and dissipation (the oracle's diag) every 10 steps.
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

STEPS = 500
SEED, AMP, NOISE = 2024, 0.05, 1e-4
PROBES = [(0, 0, 0), (2, 1, 3), (5, 7, 24), (10, 3, 25), (64, 100, 50), (33, 200, 99), (128, 17, 100),
          (200, 255, 150), (257, 0, 199), (1, 128, 120), (7, 64, 75), (99, 99, 99), (31, 5, 1), (150, 42, 175),
          (222, 222, 60), (3, 250, 198)]  # (i, j, k) into (nxpp, ny, nz)


def fingerprint(state):
    rng = np.random.default_rng(7)
    ref = rng.standard_normal(state.shape)
    out = {}
    for q, name in enumerate("uvwr"):
        f = state[q]
        out[name] = {"norm": float(np.linalg.norm(f)), "dot": float(np.sum(f * ref[q])),
                     "probes": [float(f[k, j, i]) for (i, j, k) in PROBES]}
    return out


def main():
    import oracle
    from iwrepo_b200 import config as cf
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else STEPS
    oracle.set_threads(int(sys.argv[2]) if len(sys.argv) > 2 else oracle.max_threads())
    out = sys.argv[3] if len(sys.argv) > 3 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                              "c2_fingerprint.json")
    cfg = cf.baseline("C2")
    o = oracle.Oracle(cfg)
    o.init_mode1(AMP, NOISE, SEED)
    series = []
    t0 = time.time()
    for chunk in range(steps // 10):
        o.step(10)
        d = o.diag()
        series.append({"step": 10 * (chunk + 1), "ke": float(d["ke"]), "eps": float(d["eps"])})
        print(series[-1], round(time.time() - t0), "s", flush=True)
    res = {"config": "C2", "steps": steps, "seed": SEED, "amp": AMP, "noise": NOISE,
           "fields": fingerprint(o.state(0)), "series": series,
           "_about": "oracle (FP64 CPU restatement), tests/golden/make_c2_fingerprint.py"}
    with open(out, "w") as f:
        json.dump(res, f, indent=0)


if __name__ == "__main__":
    main()
