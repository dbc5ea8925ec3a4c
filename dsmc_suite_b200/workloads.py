"""Synthetic workloads of the benchmark configurations and the derived quantities their reports
use (physical number density, column density, the two-phase collisional pipeline).

Nothing here runs particles on the host: problems are built as parameter structs and surface
arrays, and solved by the CUDA library through Context or Server.

Workloads (seeded; the shapes and distributions of the published configurations):
  * batch_instances: 64 independent ballistic exospheres; particle counts lognormal with median
    3e5 and sigma_ln 1.17, clipped to [1e4, 1e7]; body uniform over Ceres (R 470 km,
    GM 6.26e10), Europa (1561 km, 3.20e12) and Moon (1737 km, 4.90e12); sub-solar temperature
    U(100, 400) K on T = max(110 K, T_ss cos(z)^0.25); sub-solar longitude uniform; 20-60 shells.
  * served_stream: Poisson arrivals, each request drawn like a batch instance, 70 % ballistic and
    30 % collisional, each with its own seed.
  * two_phase: phase 1 collisionless with per-cell speed histograms, the degree-6 FP64 CDF fit
    per cell, the background number density from the weighted residence times, then phase 2 with
    hard-sphere collisions (d = 4.6e-10 m) against partners drawn from the fits.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

BODIES = {"ceres": (470e3, 6.26e10), "europa": (1561e3, 3.20e12), "moon": (1737e3, 4.90e12)}
D_H2O = 4.6e-10
M_H2O = 2.99e-26


@dataclass
class Problem:
    """One solve: parameters, surface arrays, optional collision tables and particle count."""
    name: str
    params: N.Params
    surface: N.SurfaceInputs
    n: int
    collision: N.CollisionInputs | None = None
    meta: dict = field(default_factory=dict)


_ICO: N.Icosphere | None = None


def icosphere() -> N.Icosphere:
    global _ICO
    if _ICO is None:
        _ICO = N.Icosphere(3)
    return _ICO


def sun_vector(lon: float) -> np.ndarray:
    return np.array([math.cos(lon), math.sin(lon), 0.0])


def config_surface(sun=(1.0, 0.0, 0.0), T_ss: float = 235.0, flux_weighted: bool = False):
    """Icosphere surface with T = max(110 K, T_ss cos(z)^0.25); optionally the launch face
    chosen in proportion to the Antoine sublimation flux (then also returns the production rate
    of a unit-radius body, molecules/s per m^2 of R^2)."""
    ico = icosphere()
    T = ico.face_temperature(sun=sun, T_ss=T_ss, T_floor=110.0)
    if flux_weighted:
        cdf, rate = ico.source_cdf(T, M_H2O)
        return N.SurfaceInputs(ico=ico, face_T=T, face_cdf=cdf), rate
    return N.SurfaceInputs(ico=ico, face_T=T)


def lognormal_count(rng: np.random.Generator, median=3e5, sigma=1.17, lo=1e4, hi=1e7) -> int:
    return int(np.clip(round(median * math.exp(sigma * rng.standard_normal())), lo, hi))


def random_instance(rng: np.random.Generator, k: int, runner: int = N.RUNNER_BALLISTIC,
                    hd: int | None = None) -> Problem:
    body = list(BODIES)[int(rng.integers(0, 3))]
    R, GM = BODIES[body]
    T_ss = float(rng.uniform(100.0, 400.0))
    lon = float(rng.uniform(0.0, 2 * math.pi))
    hd = int(rng.integers(20, 61)) if hd is None else hd
    seed = int(rng.integers(1, 2**63))
    p = N.params_config(runner, R, GM, hd, seed)
    s = sun_vector(lon)
    p.sun[0], p.sun[1], p.sun[2] = s
    surf = config_surface(s, T_ss)
    return Problem(f"{body}-{k}", p, surf, lognormal_count(rng),
                   meta={"body": body, "T_ss": T_ss, "lon": lon, "hd": hd, "seed": seed})


def batch_instances(seed: int = 20261203, count: int = 64) -> list[Problem]:
    rng = np.random.default_rng(seed)
    return [random_instance(rng, k) for k in range(count)]


# ------------------------------------------------------------------------------------------
# Grid geometry and derived quantities (FP64 on the host, from device-accumulated sums)


def shell_radii(p: N.Params) -> np.ndarray:
    """Shell boundaries r_0 = R ... r_hd = max_height (grid.c:41-99 geometry)."""
    j = np.arange(p.hd + 1, dtype=np.float64)
    if p.use_exp_grid:
        return p.Radii + p.unih * ((1.0 + p.alpha2) ** j - 1.0) / p.alpha2
    return p.Radii + j * p.unih


def cell_volumes(p: N.Params) -> np.ndarray:
    """Physical cell volumes [hd][ftd][ffd] (r_o^3 - r^3)/3 * dphi * |sin b_o - sin b|."""
    r = shell_radii(p)
    b = np.arange(p.ftd + 1) / p.ftd * math.pi - math.pi / 2
    dr3 = (r[1:] ** 3 - r[:-1] ** 3) / 3.0
    ds = np.abs(np.sin(b[1:]) - np.sin(b[:-1]))
    dphi = 2 * math.pi / p.ffd
    return dr3[:, None, None] * ds[None, :, None] * dphi * np.ones((1, 1, p.ffd))


def number_density(p: N.Params, density_fixed: np.ndarray, n: int, rate: float) -> np.ndarray:
    """Number density [m^-3] per cell from the fixed-point weight-step sums: each of the n test
    particles stands for rate / n molecules/s, and one weight-step is dt seconds of residence."""
    w = density_fixed.astype(np.float64).reshape(p.hd, p.ftd, p.ffd) / N.FIXED_SCALE
    return w * (rate / n) * p.dt_step / cell_volumes(p)


def column_density(p: N.Params, nden: np.ndarray, b_over_R) -> np.ndarray:
    """Column density [m^-2] of the shell-averaged density along lines of sight at impact
    parameters b (in body radii): exact for densities constant within each shell."""
    r = shell_radii(p)
    vol = cell_volumes(p).reshape(p.hd, -1)
    shell = (nden.reshape(p.hd, -1) * vol).sum(1) / vol.sum(1)
    out = []
    for bR in np.atleast_1d(b_over_R):
        b = bR * p.Radii
        lo = np.sqrt(np.maximum(r[:-1] ** 2 - b * b, 0.0))
        hi = np.sqrt(np.maximum(r[1:] ** 2 - b * b, 0.0))
        out.append(float(2.0 * np.sum(shell * (hi - lo))))
    return np.array(out)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# ------------------------------------------------------------------------------------------
# Two-phase collisional pipeline (dsmc then dsmc-adv of the reference, config model)


def fit_layout(p: N.Params, a: np.ndarray) -> np.ndarray:
    """Reorders per-cell rows from the density layout [ht][td][fd] to the fit layout
    [td][fd][ht] the collision tables use (advanced.c:41)."""
    return a.reshape(p.hd, p.ftd, p.ffd, -1).transpose(1, 2, 0, 3).reshape(p.hd * p.ftd * p.ffd, -1)


def two_phase_tables(ctx, p1: N.Params, surf: N.SurfaceInputs, n1: int, rate: float,
                     degree: int = 6, path: int = N.PATH_FAST_FP32, nbins: int = 64,
                     bin_width: float = 25.0):
    """Phase 1 on the GPU with per-cell speed histograms, then the FP64 fits on the device.
    Returns (CollisionInputs, phase-1 density in m^-3)."""
    p = p1.copy()
    p.runner = N.RUNNER_BALLISTIC
    p.n_speed_bins = nbins
    p.speed_bin_width = bin_width
    ctx.setup(p, surf)
    ctx.zero()
    ctx.run(path, 0, n1)
    ctx.sync()
    hist = ctx.speed_hist()
    nden = number_density(p, ctx.density(), n1, rate)
    coef, box, total, valid = ctx.fit_hist(hist, bin_width, degree)
    col = N.CollisionInputs(nden.ravel(), fit_layout(p, coef), fit_layout(p, box),
                            fit_layout(p, total[:, None]).ravel(),
                            fit_layout(p, valid[:, None]).ravel(), degree)
    return col, nden


# Total water production of the collisional problems [molecules/s]: Ceres' observed ~6 kg/s.
# The Antoine sublimation flux of a fully icy surface at these temperatures would be ~1e33/s, a
# near-surface mean free path below a millimetre, where a test-particle scheme (collisions against
# a fixed background) no longer applies; the flux sets where particles start, this rate sets how
# many molecules each test particle stands for, hence the background density of phase 2.
PRODUCTION_RATE = 2.0e26


def collisional_problem(ctx, name: str, R: float, GM: float, hd: int, seed: int, sun, T_ss: float,
                        n1: int, n2: int, path: int = N.PATH_FAST_FP32,
                        production_rate: float | None = PRODUCTION_RATE) -> Problem:
    """A config-model collisional problem: Antoine-flux source on the T map, phase-1 tables.
    production_rate None keeps the full Antoine rate of an all-ice surface."""
    surf, rate_r2 = config_surface(sun, T_ss, flux_weighted=True)
    antoine_rate = rate_r2 * R * R
    rate = antoine_rate if production_rate is None else production_rate
    p = N.params_config(N.RUNNER_ADVANCED, R, GM, hd, seed)
    p.sun[0], p.sun[1], p.sun[2] = sun
    p.cross_section = math.pi * D_H2O * D_H2O
    col, nden = two_phase_tables(ctx, p, surf, n1, rate, path=path)
    return Problem(name, p, surf, n2, col, meta={"rate": rate, "antoine_rate": antoine_rate,
                                                   "n_phase1": n1, "max_n_bg": float(nden.max())})


def served_stream(ctx, rate_hz: float, seconds: float, seed: int = 20261203,
                  collisional_frac: float = 0.3, n_tables: int = 6):
    """Poisson arrival times and requests. Collisional requests draw from n_tables phase-1
    table sets prepared here (one per body and temperature class, 50 shells)."""
    rng = np.random.default_rng(seed)
    tables = []
    for k in range(n_tables):
        body = list(BODIES)[k % 3]
        R, GM = BODIES[body]
        T_ss = 180.0 if k < 3 else 320.0
        lon = float(rng.uniform(0, 2 * math.pi))
        tables.append(collisional_problem(ctx, f"tables-{body}-{int(T_ss)}", R, GM, 50,
                                          int(rng.integers(1, 2**63)), sun_vector(lon), T_ss,
                                          200_000, 0))
    t, out = 0.0, []
    k = 0
    while True:
        t += float(rng.exponential(1.0 / rate_hz))
        if t > seconds:
            break
        if rng.uniform() < collisional_frac:
            base = tables[int(rng.integers(0, n_tables))]
            p = base.params.copy()
            p.seed = int(rng.integers(1, 2**63))
            req = Problem(f"col-{k}", p, base.surface, lognormal_count(rng), base.collision,
                          meta={"kind": "collisional", "table": base.name})
        else:
            req = random_instance(rng, k)
            req.meta["kind"] = "ballistic"
        out.append((t, req))
        k += 1
    return out


# ------------------------------------------------------------------------------------------
# Synthetic body mesh for the shadow-flux model (no mesh files ship with the reference)


def cratered_mesh(nlevel: int = 4, craters: int = 16, depth: float = 0.15, width: float = 0.25,
                  seed: int = 20261203, radius: float = 1.0):
    """Icosphere of 20 * 4^nlevel faces with Gaussian craters pressed into it (concave, so faces
    shadow each other at low sun). Returns (spot [npoint][3], facet [nface][3] 0-based)."""
    ico = N.Icosphere(nlevel)
    fv = ico.face_verts.reshape(-1, 3)
    key = np.round(fv, 12)
    uniq, inv = np.unique(key, axis=0, return_inverse=True)
    spot = uniq.astype(np.float64)
    facet = inv.reshape(-1, 3).astype(np.int32)
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(craters, 3))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    u = spot / np.linalg.norm(spot, axis=1, keepdims=True)
    d2 = ((u[:, None, :] - c[None, :, :]) ** 2).sum(-1)
    r = radius * (1.0 - depth * np.exp(-d2 / (width * width)).sum(1).clip(max=1.0))
    return u * r[:, None], facet
