"""Generates tests/golden/reference_thermal.npz: surface temperatures computed by the reference's
own thermal_solve (src/thermal/thermal_model.c, compiled from its sources into oracle/_ref by
oracle/Makefile) for three cases - default Ceres parameters with the analytic flux, a seeded
random flux, and a short shallow column - so the oracle can be pinned where the reference build
is absent. Run from the repository root: python tests/golden/make_thermal_golden.py"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def cases(N):
    """(name, ftd, ffd, ThermalParams, flux or None)."""
    out = [("default", 36, 72, N.ThermalParams.default(), None)]
    rng = np.random.default_rng(20261203)
    flux = rng.uniform(0.0, 250.0, (18, 24)) * (rng.uniform(size=(18, 24)) > 0.2)
    out.append(("random_flux", 18, 24, N.ThermalParams.default(), flux))
    tp = N.ThermalParams.default()
    tp.n_substep = 2
    tp.depth = 0.002
    tp.albedo = 0.1
    out.append(("shallow", 12, 16, tp, None))
    return out


def main():
    from dsmc_suite_b200 import _native as N
    from oracle import oracle as O
    O.build()
    res = {}
    for name, ftd, ffd, tp, flux in cases(N):
        T = O.reference_thermal(ftd, ffd, tp, flux)
        if T is None:
            raise SystemExit("oracle/_ref/libdsmcref.so is missing: build it with make -C oracle ref")
        res[name] = T
        if flux is not None:
            res[name + "_flux"] = flux
    np.savez(ROOT / "tests" / "golden" / "reference_thermal.npz", **res)


if __name__ == "__main__":
    main()
