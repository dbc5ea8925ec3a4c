"""The FAST paths against the FP64 paths that the oracle pins (needs a B200).

Chain of references: the oracle reproduces the reference binary byte for byte (rand_r mode) and,
on the kernels' Philox streams, PLAIN_FP64 reproduces the oracle (test_gpu_parity.py). Here:
  * FAST_FP64 (the resident-slot engine on FP64 state) against PLAIN_FP64 and the oracle on the
    same streams: the same particles end the same way after the same number of steps, and the
    grids differ only where FP64 rounding moved a step across a cell boundary;
  * FAST_FP32 against PLAIN_FP64 on the loops and bodies the FP32 engine runs - the config-model
    collisional lean loop with degree-6 fits, the Europa- and Moon-like bodies - with fates equal,
    collision counts within 1 % and a density relative L2 below a stated fraction of the Monte
    Carlo noise between two independent FP64 runs;
  * FAST_FP32 against FAST_FP64 at the full Ceres-like size of 1e8 particles, where no other
    FP64 path finishes in seconds: density relative L2 <= 1e-3, the accuracy bar of the FP32 push;
  * the per-hop energy-drift guard: no hop of the config workloads is flagged at dt = 2 s, and at
    an oversized step every path flags about the hops the oracle flags.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import cold_T

pytestmark = pytest.mark.gpu

BODIES = {"ceres": (470e3, 6.26e10), "europa": (1561e3, 3.20e12), "moon": (1737e3, 4.90e12)}


@pytest.fixture(scope="module")
def surface(N):
    ico = N.Icosphere(3)
    return N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _noise(ctx, N, p, S, n, col=None):
    """Density relative L2 between two independent PLAIN_FP64 runs (other seeds)."""
    q1, q2 = p.copy(), p.copy()
    q1.seed, q2.seed = p.seed + 1001, p.seed + 2002
    a = ctx.solve(N.PATH_PLAIN_FP64, q1, S, n, collision=col)["density"]
    b = ctx.solve(N.PATH_PLAIN_FP64, q2, S, n, collision=col)["density"]
    return _rel(a, b)


@pytest.fixture(scope="module")
def collisional(ctx, N):
    """The config-model collisional workload of the two-phase solve: Antoine-flux source, phase 1
    of 1e5 particles with 64-bin speed histograms, degree-6 FP64 fits, production 2e26 /s."""
    from dsmc_suite_b200 import workloads as W
    return W.collisional_problem(ctx, "collisional", 470e3, 6.26e10, 50, 20261203,
                                 W.sun_vector(0.0), 235.0, 100_000, 100_000,
                                 path=N.PATH_PLAIN_FP64)


def _cases(N, surface, collisional):
    out = {}
    for body, (R, GM) in BODIES.items():
        out[body] = (N.params_config(N.RUNNER_BALLISTIC, R, GM, 50, 20261203), surface, None, 100_000)
    out["reference"] = (N.params_reference(N.RUNNER_BALLISTIC, 36, 72), N.SurfaceInputs(T_map=cold_T(N)),
                        None, 30_000)
    P = collisional
    out["collisional"] = (P.params, P.surface, P.collision, P.n)
    return out


@pytest.mark.parametrize("case", ["ceres", "europa", "moon", "reference", "collisional"])
def test_fast_fp64_follows_plain_fp64(ctx, N, surface, collisional, case):
    p, S, col, n = _cases(N, surface, collisional)[case]
    a = ctx.solve(N.PATH_PLAIN_FP64, p, S, n, collision=col, outputs=True)
    b = ctx.solve(N.PATH_FAST_FP64, p, S, n, collision=col, outputs=True)
    same = (a["fate"] == b["fate"]) & (a["steps"] == b["steps"])
    assert same.mean() >= 0.99, same.mean()
    sa, sb = a["stats"], b["stats"]
    assert abs(sb["total_steps"] / sa["total_steps"] - 1) < 1e-3
    assert sb["n_finished"] == sa["n_finished"] == n
    if col is not None:
        assert sa["n_collisions"] > 1000
        assert abs(sb["n_collisions"] / sa["n_collisions"] - 1) < 0.01
    rel = _rel(b["density"], a["density"])
    noise = _noise(ctx, N, p, S, n, col)
    assert rel < 0.1 * noise, (rel, noise)


def test_fast_fp64_vs_oracle(ctx, N, O, surface):
    p = N.params_config(N.RUNNER_BALLISTIC)
    n = 3000
    g = ctx.solve(N.PATH_FAST_FP64, p, surface, n, outputs=True)
    o = O.run(p, surface, n, nthreads=4)
    same = (g["fate"] == o["fate"]) & (g["steps"] == o["steps"])
    assert same.mean() >= 0.99, same.mean()
    assert g["stats"]["total_steps"] == pytest.approx(o["total_steps"], rel=1e-3)
    assert np.abs(g["density"].astype(float) - o["density"]).sum() <= 0.01 * o["density"].sum()


@pytest.mark.parametrize("case", ["collisional", "europa", "moon"])
def test_fast_fp32_vs_plain_fp64_lean_loops(ctx, N, surface, collisional, case):
    """The FP32 engine's lean loops against the FP64 path on the same streams: the collisional
    loop (isotropic hard spheres against degree-6 fitted CDFs) and the relaunch-bound bodies."""
    p, S, col, n = _cases(N, surface, collisional)[case]
    a = ctx.solve(N.PATH_PLAIN_FP64, p, S, n, collision=col, outputs=True)
    b = ctx.solve(N.PATH_FAST_FP32, p, S, n, collision=col, outputs=True)
    assert np.mean(a["fate"] == b["fate"]) >= 0.99
    sa, sb = a["stats"], b["stats"]
    assert abs(sb["total_steps"] / sa["total_steps"] - 1) < 0.01
    if col is not None:
        assert sa["n_collisions"] > 1000
        assert abs(sb["n_collisions"] / sa["n_collisions"] - 1) < 0.01
    rel = _rel(b["density"], a["density"])
    noise = _noise(ctx, N, p, S, n, col)
    assert rel < 0.25 * noise, (rel, noise)


def test_full_size_ceres_fast_fp32_vs_fast_fp64(ctx, N, surface):
    """1e8 particles of the Ceres-like workload: the FP32 compensated path against the FP64
    engine on the same streams, density relative L2 <= 1e-3; horizon grid and step count too."""
    p = N.params_config(N.RUNNER_BALLISTIC)
    n = 100_000_000
    ctx.setup(p, surface)
    res = {}
    for path in (N.PATH_FAST_FP64, N.PATH_FAST_FP32):
        ctx.zero()
        ctx.run(path, 0, n)
        ctx.sync()
        res[path] = (ctx.density(), ctx.horizon(), ctx.stats())
    d64, h64, s64 = res[N.PATH_FAST_FP64]
    d32, h32, s32 = res[N.PATH_FAST_FP32]
    assert s32["n_finished"] == s64["n_finished"] == n
    assert _rel(d32, d64) <= 1e-3
    assert _rel(h32, h64) <= 1e-3
    assert abs(s32["total_steps"] / s64["total_steps"] - 1) < 1e-4


def test_energy_drift_guard_on_every_path(ctx, N, O, surface):
    """No hop of the config workload drifts beyond drift_tol * GM / R at dt = 2 s; at dt = 20 s
    the integrator's first-order velocity update drifts past it and every path flags about the
    hops the oracle flags (the plain FP64 path the same count up to last-place differences)."""
    for body in ("ceres", "moon"):
        R, GM = BODIES[body]
        p = N.params_config(N.RUNNER_BALLISTIC, R, GM, 50, 20261203)
        for path in (N.PATH_PLAIN_FP64, N.PATH_FAST_FP64, N.PATH_FAST_FP32):
            assert ctx.solve(path, p, surface, 20_000)["stats"]["n_drift_flagged"] == 0, (body, path)
        p.dt_step = 20.0
        p.wdecay = math.exp(-p.dt_step / p.lifetime)
        n = 3000
        o = O.run(p, surface, n, nthreads=4, particles=False)["n_drift_flagged"]
        assert o > 1000
        got = {path: ctx.solve(path, p, surface, n)["stats"]["n_drift_flagged"]
               for path in (N.PATH_PLAIN_FP64, N.PATH_FAST_FP64, N.PATH_FAST_FP32)}
        assert abs(got[N.PATH_PLAIN_FP64] - o) <= max(3, 0.002 * o), (got, o)
        for path in (N.PATH_FAST_FP64, N.PATH_FAST_FP32):
            assert abs(got[path] - o) <= 0.03 * o, (body, path, got, o)
        p.drift_tol = 0.0
        assert ctx.solve(N.PATH_FAST_FP32, p, surface, 500)["stats"]["n_drift_flagged"] == 0
