"""Reader for `<prefix>_grids.bin`, the binary side-car the runners write with DSMC_SIDECAR=1
(the CLI's `--bin`).

The reference's text outputs print density to 6 decimals (`%9.6f`, src/common/fileio.c:27-45)
and per-particle rows to 5 (`%9.5f`, fileio.c:111-123), so a file-level comparison stops at
1e-6. The side-car holds what those files round: the fixed-point density and horizon grids
(count / fixed_scale is the printed value) and the FP64 rows, in the files' own order. Layout,
little-endian: 8-byte magic "DSMCBIN1"; int32 ftd, ffd, hd, nrows; int64 totaln; float64
fixed_scale; uint64 den[hd * ftd * ffd]; uint64 horizon[ftd * ffd]; float64 ttime[nrows *
totaln]."""
from __future__ import annotations

from pathlib import Path

import numpy as np

MAGIC = b"DSMCBIN1"
_HEADER = np.dtype([("magic", "S8"), ("ftd", "<i4"), ("ffd", "<i4"), ("hd", "<i4"),
                    ("nrows", "<i4"), ("totaln", "<i8"), ("fixed_scale", "<f8")])


def read_grids_bin(path: str | Path) -> dict:
    """Return {ftd, ffd, hd, nrows, totaln, fixed_scale, density (uint64, flat in _den.dat
    order), horizon (uint64, flat), ttime (float64, shape (nrows, totaln))}. Raises ValueError on
    a wrong magic number or a file whose length does not match its header."""
    raw = Path(path).read_bytes()
    if len(raw) < _HEADER.itemsize:
        raise ValueError(f"{path}: shorter than the side-car header")
    h = np.frombuffer(raw, _HEADER, count=1)[0]
    if bytes(h["magic"]) != MAGIC:
        raise ValueError(f"{path}: not a grids side-car (magic {bytes(h['magic'])!r})")
    ftd, ffd, hd, nrows, totaln = (int(h[k]) for k in ("ftd", "ffd", "hd", "nrows", "totaln"))
    ncell, nh, nt = hd * ftd * ffd, ftd * ffd, nrows * max(totaln, 0)
    want = _HEADER.itemsize + 8 * (ncell + nh + nt)
    if min(ftd, ffd, hd, nrows) < 0 or len(raw) != want:
        raise ValueError(f"{path}: {len(raw)} bytes, header implies {want}")
    off = _HEADER.itemsize
    den = np.frombuffer(raw, "<u8", ncell, off)
    hor = np.frombuffer(raw, "<u8", nh, off + 8 * ncell)
    tt = np.frombuffer(raw, "<f8", nt, off + 8 * (ncell + nh)).reshape(nrows, max(totaln, 0))
    return {"ftd": ftd, "ffd": ffd, "hd": hd, "nrows": nrows, "totaln": totaln,
            "fixed_scale": float(h["fixed_scale"]), "density": den.copy(), "horizon": hor.copy(),
            "ttime": tt.copy()}
