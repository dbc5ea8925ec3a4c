"""The thermal column model on the GPU against the oracle (needs a B200).

The oracle is pinned bit for bit to the reference's thermal_solve (test_oracle_golden.py). The
GPU follows the same FP64 operation order (-fmad=false), so its Crank-Nicolson and Thomas steps
are exact; CUDA's log10 / pow / sqrt inside the surface energy balance may round differently in
the last place from glibc's, which can move a bisection bracket by one halving. Bar: at least
99 % of the cells bit-identical and every cell within 0.02 K (twice the bisection tolerance)."""
from __future__ import annotations

import ctypes as C
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _cases(N):
    from test_oracle_golden import _thermal_cases
    return _thermal_cases(N)


def _close(g, o):
    assert np.mean(g == o) >= 0.99, np.mean(g == o)
    assert np.abs(g - o).max() <= 0.02, np.abs(g - o).max()


def test_thermal_matches_oracle(ctx, N, O):
    for name, ftd, ffd, tp, flux in _cases(N):
        T, h = ctx.thermal(ftd, ffd, tp, flux)
        To, ho = O.thermal(ftd, ffd, tp, flux)
        assert h == ho
        _close(T, To)


def test_kept_thermal_solve_entry_point(N, O):
    """thermal_solve(grid, params, flux, nthreads) with the reference's signature and structs."""
    tp = N.ThermalParams.default()
    T = np.zeros((36, 72))
    g = N.SphericalGrid(ftd=36, ffd=72, hd=1, temperature=T.ctypes.data_as(C.POINTER(C.c_double)))
    N.lib().thermal_solve(C.byref(g), C.byref(tp), None, 4)
    _close(T, O.thermal(36, 72, tp)[0])


def test_cli_thermal_and_pipeline(N, O, tmp_path, built):
    cli = ROOT / "dsmc_suite_b200" / "bin" / "dsmc_suite"
    r = subprocess.run([str(cli), "thermal", "-o", str(tmp_path / "t")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    assert "Thermal model: dr=" in r.stdout and "Thermal model done." in r.stdout
    vals = (tmp_path / "t_temperature.dat").read_text().split()
    assert vals[:2] == ["36", "72"]
    T = np.array(vals[2:], dtype=np.float64).reshape(36, 72)
    ref = np.array(["%8.6f" % x for x in O.thermal(36, 72, N.ThermalParams.default())[0].ravel()],
                   dtype=np.float64).reshape(36, 72)
    assert np.abs(T - ref).max() <= 0.02
    r = subprocess.run([str(cli), "pipeline", "-n", "300", "-o", str(tmp_path / "p")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for f in ("p_temperature.dat", "p_phase1_den.dat", "p_phase1_v_record.dat",
              "p_phase2_den.dat", "p_phase2_ttime.dat"):
        assert (tmp_path / f).exists(), f
    assert "PIPELINE COMPLETE" in r.stdout


def test_thermal_edge_cases(ctx, N, O):
    """Smallest grid and column (3 depth points), one step, a night-only flux, and the
    argument checks."""
    tp = N.ThermalParams.default()
    tp.depth = 1e-6
    tp.n_substep = 1
    T, h = ctx.thermal(1, 2, tp)
    To, ho = O.thermal(1, 2, tp)
    assert h == ho == 3
    _close(T, To)
    flux = np.zeros((4, 6))
    T, _ = ctx.thermal(4, 6, N.ThermalParams.default(), flux)
    _close(T, O.thermal(4, 6, N.ThermalParams.default(), flux)[0])
    bad = N.ThermalParams.default()
    bad.n_substep = 0
    with pytest.raises(N.DsmcError):
        ctx.thermal(4, 6, bad)
    with pytest.raises(N.DsmcError):
        ctx.thermal(0, 6, N.ThermalParams.default())
