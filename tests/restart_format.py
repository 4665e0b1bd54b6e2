"""Independent reader of restart files for the tests: ifort unformatted
sequential framing (4-byte little-endian byte count before and after each
record) and the record list of output.f:26-108 (REAL*8 and INTEGER*4 items)."""
import struct

import numpy as np


def records(path):
    """All records of a file as bytes objects; raises on bad framing."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        assert 0 <= n and pos + 8 + n <= len(data), "bad leading byte count"
        (n2,) = struct.unpack_from("<i", data, pos + 4 + n)
        assert n2 == n, "trailing byte count differs"
        out.append(data[pos + 4: pos + 4 + n])
        pos += 8 + n
    return out


def layout(cfg):
    """(REAL*8 items, INTEGER*4 items) of each of output.f's 49 records."""
    nx, ny, nz, N, ns = cfg.nx, cfg.ny, cfg.nz, cfg.nzloc, cfg.nsubd
    nxpp, nz2, nt = nx + 2, ns * (N - 1) + 1, (nx + 2) * ny * nz
    lay = [(1, 0), (2, 0), (0, 9), (2, 0), (2 * nx, 0), (2 * ny, 0), (nx, 0), (ny, 0), (nz, 0), (nz2, 0),
           (2 * ns, ns), (1, 0), (N * N, 0), (N * N, 0), (N, 0), (N, 0), (N * N, 0), (N * N, 0), (N * N, 0),
           (3 * nz, 0), (2 * nxpp * ny, 0), (3 * 2 * nxpp * ny * 2, 0), (1, 0), (1, 0)]
    lay += [(2 * nxpp * nz, 0)] * 3 + [(nxpp * nz, 0), (2 * nxpp * nz, 0)]
    lay += [(nt, 0)] * 20
    return lay


def f8(rec):
    return np.frombuffer(rec, dtype="<f8")


def state_levels(recs, cfg):
    """Records 30-49 as the (5, 4, nz, ny, nxpp) levels n, n-1, n-2, NL n-1, NL n-2."""
    shp = (cfg.nz, cfg.ny, cfg.nxpp)
    return np.stack([np.stack([f8(recs[29 + 4 * lv + q]).reshape(shp) for q in range(4)]) for lv in range(5)])


def extra(recs):
    """The continuation record: (istep, ivardt, idtstep, istart), (dt, cdt, fac1..3, bdf1..3, bdfv)."""
    r = recs[49]
    ints = struct.unpack_from("<6i", r, 0)
    assert ints[0] == 0x32425749 and ints[1] == 1
    return ints[2:], struct.unpack_from("<9d", r, 24)
