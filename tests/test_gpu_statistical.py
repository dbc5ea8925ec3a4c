"""Statistical parity of the GPU paths with the reference CPU run (needs a B200).

The GPU draws Philox streams and the reference draws glibc rand_r, so their fields agree only
within Monte Carlo noise. The reference run here is the oracle in rand_r mode, which reproduces
the reference binary's `dsmc -t 1` output files byte for byte (test_oracle_golden.py).

Both sides run B independent batches (seeds); under the null hypothesis the 2B batches are
exchangeable, so each statistic's p-value comes from random re-splits of the batches into two
groups (a permutation test, valid for the weighted, particle-correlated residence sums):
  * per-cell chi-square: sum over populated cells of (mean_a - mean_b)^2 / (var_a + var_b);
  * Kolmogorov-Smirnov distance between the radial (per-shell) density profiles;
  * speed distribution of the velocity records (KS distance of the pooled speed samples).
Bar: p > 0.01 for each."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cold_T

pytestmark = pytest.mark.gpu

B = 48          # batches per side
M = 2000        # particles per batch
PERMS = 400


def _chi2(a: np.ndarray, b: np.ndarray) -> float:
    ma, mb = a.mean(0), b.mean(0)
    v = a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b)
    m = v > 0
    return float(np.sum((ma[m] - mb[m]) ** 2 / v[m]))


def _ks(a: np.ndarray, b: np.ndarray) -> float:
    """KS distance of the pooled profiles (rows = batches, columns = ordered bins)."""
    pa, pb = np.cumsum(a.sum(0)), np.cumsum(b.sum(0))
    return float(np.max(np.abs(pa / pa[-1] - pb / pb[-1])))


def _perm_pvalue(a: np.ndarray, b: np.ndarray, stat, seed: int = 7) -> tuple[float, float]:
    obs = stat(a, b)
    pool = np.concatenate([a, b])
    rng = np.random.default_rng(seed)
    ge = 0
    for _ in range(PERMS):
        idx = rng.permutation(len(pool))
        ge += stat(pool[idx[:len(a)]], pool[idx[len(a):]]) >= obs
    return obs, (ge + 1) / (PERMS + 1)


def _gpu_batches(ctx, N, p, S, path, col=None):
    out = []
    for k in range(B):
        q = p.copy()
        q.seed = 1000 + k
        r = ctx.solve(path, q, S, M, collision=col)
        out.append(r["density"].astype(np.float64).ravel() / N.FIXED_SCALE)
    return np.array(out)


def _reference_batch(args):
    """One reference batch (runs in a spawned worker: rand_r mode is single-threaded)."""
    import sys
    from pathlib import Path
    root = str(Path(__file__).resolve().parents[1])
    if root not in sys.path:
        sys.path.insert(0, root)
    from dsmc_suite_b200 import _native as N
    from oracle import oracle as O
    kind, k, extra = args
    if kind == "ballistic":
        p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
        S = N.SurfaceInputs(T_map=extra)
        col = None
    else:
        p, col, T = extra
        p = N.Params.from_buffer_copy(p)
        col = N.CollisionInputs(*col)
        S = N.SurfaceInputs(T_map=T)
    r = O.run(p, S, M, collision=col, rng=O.RNG_RAND_R, rr_seed=5000 + 17 * k, fixed=False,
              f64=True, nthreads=1)
    return np.asarray(r["density_f64"], dtype=np.float64).ravel()


def _reference_batches(kind, extra):
    import multiprocessing as mp
    import os
    with mp.get_context("spawn").Pool(min(B, os.cpu_count() or 1)) as pool:
        return np.array(pool.map(_reference_batch, [(kind, k, extra) for k in range(B)]))


@pytest.fixture(scope="module")
def reference_ballistic(N, O):
    p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    T = cold_T(N)
    return p, N.SurfaceInputs(T_map=T), _reference_batches("ballistic", T)


def _coarse(x: np.ndarray, hd: int) -> np.ndarray:
    """Sums of 3 x 6 (latitude x longitude) cell blocks within each shell."""
    return x.reshape(len(x), hd, 12, 3, 12, 6).sum((3, 5)).reshape(len(x), -1)


def _field_pvalues(a, b, hd):
    """p-values of the per-cell and per-block chi-squares (over cells populated in every batch)
    and of the radial-profile KS distance."""
    out = {}
    for name, (x, y) in (("cells", (a, b)), ("blocks", (_coarse(a, hd), _coarse(b, hd)))):
        mask = (x > 0).all(0) & (y > 0).all(0)
        assert mask.sum() > 100
        out[name] = _perm_pvalue(x[:, mask], y[:, mask], _chi2)
    radial = lambda x: x.reshape(len(x), hd, -1).sum(2)
    out["radial_ks"] = _perm_pvalue(radial(a), radial(b), _ks)
    return out


def _check_fields(a, b, hd):
    for name, (stat, pval) in _field_pvalues(a, b, hd).items():
        assert pval > 0.01, (name, stat, pval)


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_ballistic_fields_match_reference_run(ctx, N, reference_ballistic, path):
    p, S, ref = reference_ballistic
    P = N.PATH_PLAIN_FP64 if path == "plain" else N.PATH_FAST_FP32
    _check_fields(_gpu_batches(ctx, N, p, S, P), ref, p.hd)


def test_permutation_test_detects_a_planted_bias(N, reference_ballistic):
    """Power check: two halves of the reference run agree, and the same statistics reject the
    second half once its southern-hemisphere weights are raised by 5 % (planted on the CPU, in
    the oracle's output)."""
    p, S, ref = reference_ballistic
    a, b = ref[: B // 2], ref[B // 2:].copy()
    assert min(pv for _, pv in _field_pvalues(a, b, p.hd).values()) > 0.01
    b = b.reshape(len(b), p.hd, p.ftd, p.ffd)
    b[:, :, : p.ftd // 2, :] *= 1.05
    assert _field_pvalues(a, b.reshape(len(b), -1), p.hd)["blocks"][1] <= 0.01


def test_advanced_fields_match_reference_run(ctx, N, O, golden):
    from test_oracle_golden import _reference_advanced_inputs
    p, col, _ = _reference_advanced_inputs(N, O, golden)
    T = golden["runs"]["T"]
    S = N.SurfaceInputs(T_map=T)
    ref = _reference_batches("advanced", (bytes(p), (col.n_bg, col.coef, col.box, col.total,
                                                      col.valid, 3), T))
    _check_fields(_gpu_batches(ctx, N, p, S, N.PATH_FAST_FP32, col), ref, p.hd)


def test_velocity_records_match_reference_speeds(ctx, N, O):
    """Speeds of the velocity records (the phase-1 statistics of dsmc-adv): GPU record pass vs
    the reference run, pooled over batches; KS distance against its permutation null."""
    p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    S = N.SurfaceInputs(T_map=cold_T(N))
    gpu, ref = [], []
    for k in range(B // 2):
        q = p.copy()
        q.seed = 3000 + k
        ctx.setup(q, S)
        v, *_ = ctx.velocity_record(M // 4)
        gpu.append(np.linalg.norm(v, axis=1))
        r = O.run(p, S, M // 4, rng=O.RNG_RAND_R, rr_seed=9000 + 31 * k, fixed=False, f64=True,
                  nthreads=1, v_record=True, particles=False)
        ref.append(np.linalg.norm(r["v_record"], axis=1))
    grid = np.linspace(0, 2000, 401)

    def hist(xs):
        return np.array([np.histogram(x, grid)[0] for x in xs], dtype=np.float64)

    d, pval = _perm_pvalue(hist(gpu), hist(ref), _ks)
    assert pval > 0.01, (d, pval)
