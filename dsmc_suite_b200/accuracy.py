"""Accuracy of the FP32 compensated path against the FP64 path on the 1e8-particle Ceres-like ballistic workload.

    python -m dsmc_suite_b200.accuracy [--particles 1e8] [--trajectories 1e4] [--md out.md]

The FP64 path is the oracle here: its push is bit-identical to the reference's verlet_step and
its solve follows the same Philox streams as the FP32 path. Reported:
  * end-point position error of fed-state trajectories: seeded launch states on the Ceres-like
    body (area-uniform surface points, flux-weighted Maxwell-Boltzmann velocities at the local
    T = max(110 K, 235 K cos(z)^0.25)), pushed by both paths up to the 20,000-step life cap or to
    landing or escape;
  * per-cell density relative L2 between the two paths on one solve of N particles, beside the
    relative L2 between two independent FP32 solves (the Monte Carlo noise at this N);
  * column density at impact parameters 1.1, 1.5, 2, 3, 5 and 8 R for both paths.
Prints one JSON line; --md also writes a markdown summary.

    python -m dsmc_suite_b200.accuracy --agreement [--particles 1e5] [--md out.md]

instead compares the three paths on the same Philox streams over five workloads (the Ceres-,
Europa- and Moon-like ballistic bodies, the reference model on a 36 x 72 map, the config-model
collisional phase 2 with degree-6 fits): per path against PLAIN_FP64, the fraction of particles
with the same fate and step count and the density relative L2, beside the relative L2 between two
independent PLAIN_FP64 runs.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import _native as N
from . import workloads as W
from .solver import Context

B_OVER_R = (1.1, 1.5, 2.0, 3.0, 5.0, 8.0)
K_B = 1.380649e-23


def launch_states(p: N.Params, m: int, seed: int = 20261203, T_ss=235.0, T_floor=110.0):
    """Seeded surface launch states (positions, velocities) [m][3] of the config model."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, m)
    ph = rng.uniform(0.0, 2 * math.pi, m)
    rho = np.sqrt(1.0 - z * z)
    n = np.stack([rho * np.cos(ph), rho * np.sin(ph), z], 1)
    cz = np.clip(n @ np.array(p.sun[:3]), 0.0, 1.0)
    T = np.maximum(T_floor, T_ss * cz ** 0.25)
    sig = np.sqrt(K_B * T / W.M_H2O)
    # flux-weighted half-space Maxwellian: Rayleigh normal component, Gaussian tangential ones
    vn = sig * np.sqrt(-2.0 * np.log1p(-rng.uniform(0.0, 1.0, m)))
    t1 = np.cross(n, np.array([0.0, 0.0, 1.0]))
    t1 /= np.maximum(np.linalg.norm(t1, axis=1, keepdims=True), 1e-30)
    t2 = np.cross(n, t1)
    g = rng.standard_normal((m, 2)) * sig[:, None]
    vel = vn[:, None] * n + g[:, :1] * t1 + g[:, 1:] * t2
    return n * p.Radii, vel


def endpoint_errors(ctx: Context, p: N.Params, surf, m: int, nsteps: int) -> dict:
    ctx.setup(p, surf)
    pos, vel = launch_states(p, m)
    P64, _, s64, t64 = ctx.push(N.PATH_PLAIN_FP64, pos, vel, nsteps)
    P32, _, s32, t32 = ctx.push(N.PATH_FAST_FP32, pos, vel, nsteps)
    same = (s64 == s32) & (t64 == t32)
    err = np.linalg.norm(P32 - P64, axis=1)
    e = err[same]
    rel = e / np.linalg.norm(P64[same], axis=1)
    return {"trajectories": m, "max_steps": nsteps, "same_outcome_frac": float(same.mean()),
            "landed": int((s64 == 1).sum()), "escaped": int((s64 == 2).sum()),
            "ran_full": int((s64 == 0).sum()), "mean_steps": float(t64.mean()),
            "err_m": {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)),
                      "max": float(e.max())},
            "err_rel": {"median": float(np.median(rel)), "p99": float(np.percentile(rel, 99)),
                        "max": float(rel.max())}}


def density_errors(ctx: Context, p: N.Params, surf, n: int) -> dict:
    t0 = time.perf_counter()
    d64 = ctx.solve(N.PATH_PLAIN_FP64, p, surf, n)
    t64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    d32 = ctx.solve(N.PATH_FAST_FP32, p, surf, n)
    t32 = time.perf_counter() - t0
    q = p.copy()
    q.seed = p.seed + 1
    d32b = ctx.solve(N.PATH_FAST_FP32, q, surf, n)
    a, b, c = (x["density"].astype(np.float64) for x in (d64, d32, d32b))
    # column densities per unit production rate (1 molecule/s), shell-averaged
    cd = {k: W.column_density(p, W.number_density(p, x["density"], n, 1.0), B_OVER_R)
          for k, x in (("fp64", d64), ("fp32", d32), ("fp32_other_seed", d32b))}
    return {"particles": n, "density_rel_l2": W.rel_l2(b, a),
            "independent_run_rel_l2": W.rel_l2(c, b),
            "ratio_to_noise": W.rel_l2(b, a) / max(W.rel_l2(c, b), 1e-300),
            "total_steps": {"fp64": d64["stats"]["total_steps"], "fp32": d32["stats"]["total_steps"]},
            "wall_s": {"fp64": t64, "fp32": t32},
            "column_density": {"b_over_R": list(B_OVER_R),
                               "fp64": cd["fp64"].tolist(), "fp32": cd["fp32"].tolist(),
                               "rel_diff": (cd["fp32"] / cd["fp64"] - 1).tolist(),
                               "independent_run_rel_diff":
                                   (cd["fp32_other_seed"] / cd["fp32"] - 1).tolist()}}


def agreement(ctx: Context, n: int) -> dict:
    """FAST_FP64 and FAST_FP32 against PLAIN_FP64 on five workloads, same Philox streams."""
    surf = W.config_surface()
    cases = []
    for body in ("ceres", "europa", "moon"):
        R, GM = W.BODIES[body]
        cases.append((body, N.params_config(N.RUNNER_BALLISTIC, R, GM, 50, 20261203), surf, None, n))
    T = N.latlon_temperature(36, 72, T_ss=235.0, T_floor=60.0)
    cases.append(("reference", N.params_reference(N.RUNNER_BALLISTIC, 36, 72), N.SurfaceInputs(T_map=T),
                  None, max(1000, n // 3)))
    prob = W.collisional_problem(ctx, "collisional", 470e3, 6.26e10, 50, 20261203, W.sun_vector(0.0),
                                 235.0, n, n, path=N.PATH_PLAIN_FP64)
    cases.append(("collisional", prob.params, prob.surface, prob.collision, n))
    out = {}
    for name, p, S, col, m in cases:
        r = {path: ctx.solve(path, p, S, m, collision=col, outputs=True)
             for path in (N.PATH_PLAIN_FP64, N.PATH_FAST_FP64, N.PATH_FAST_FP32)}
        q = p.copy()
        q.seed = p.seed + 1
        ind = ctx.solve(N.PATH_PLAIN_FP64, q, S, m, collision=col)["density"]
        a = r[N.PATH_PLAIN_FP64]
        row = {"particles": m, "noise_rel_l2": W.rel_l2(ind, a["density"]),
               "steps_plain": a["stats"]["total_steps"], "collisions_plain": a["stats"]["n_collisions"],
               "drift_flagged_plain": a["stats"]["n_drift_flagged"]}
        for path, key in ((N.PATH_FAST_FP64, "fast_fp64"), (N.PATH_FAST_FP32, "fast_fp32")):
            b = r[path]
            row[key] = {"same_fate_and_steps": float(np.mean((b["fate"] == a["fate"]) & (b["steps"] == a["steps"]))),
                        "same_fate": float(np.mean(b["fate"] == a["fate"])),
                        "density_rel_l2": W.rel_l2(b["density"], a["density"]),
                        "steps_ratio": b["stats"]["total_steps"] / max(a["stats"]["total_steps"], 1),
                        "collisions": b["stats"]["n_collisions"],
                        "drift_flagged": b["stats"]["n_drift_flagged"]}
        out[name] = row
    return out


def agreement_markdown(res: dict, cmd: str) -> str:
    rows = []
    for name, r in res.items():
        for key in ("fast_fp64", "fast_fp32"):
            x = r[key]
            rows.append(f"| {name} | {r['particles']} | {key.upper()} | {100 * x['same_fate']:.3f} % | "
                        f"{100 * x['same_fate_and_steps']:.3f} % | {x['density_rel_l2']:.2e} | "
                        f"{r['noise_rel_l2']:.2e} | {x['steps_ratio']:.6f} | {x['collisions']} "
                        f"({r['collisions_plain']}) | {x['drift_flagged']} ({r['drift_flagged_plain']}) |")
    return f"""# FAST_FP64 and FAST_FP32 against PLAIN_FP64, same Philox streams

Command: `{cmd}`

PLAIN_FP64 reproduces the oracle, which reproduces the reference binary (rand_r mode). Columns:
particles with the same fate as PLAIN_FP64; with the same fate and step count; per-cell density
relative L2 against PLAIN_FP64; the same between two independent PLAIN_FP64 runs (Monte Carlo
noise); particle-steps relative to PLAIN_FP64; collisions and drift-flagged hops (PLAIN_FP64's in
brackets).

| workload | particles | path | same fate | same fate and steps | density rel-L2 | noise rel-L2 | steps ratio | collisions | drift-flagged hops |
|---|---|---|---|---|---|---|---|---|---|
""" + "\n".join(rows) + "\n"


def markdown(res: dict, cmd: str) -> str:
    e, d = res["endpoint"], res["density"]
    cd = d["column_density"]
    rows = "\n".join(f"| {bb:g} | {f64:.4e} | {f32:.4e} | {rd:+.2e} | {nd:+.2e} |"
                     for bb, f64, f32, rd, nd in zip(cd["b_over_R"], cd["fp64"], cd["fp32"],
                                                     cd["rel_diff"], cd["independent_run_rel_diff"]))
    return f"""# FP32 compensated path vs FP64 path, 1e8-particle Ceres-like ballistic workload

Command: `{cmd}`

## End-point error, {e['trajectories']} seeded trajectories, up to {e['max_steps']} steps

| | median | p99 | max |
|---|---|---|---|
| position error [m] | {e['err_m']['median']:.3e} | {e['err_m']['p99']:.3e} | {e['err_m']['max']:.3e} |
| relative to radius | {e['err_rel']['median']:.2e} | {e['err_rel']['p99']:.2e} | {e['err_rel']['max']:.2e} |

Same outcome (status and step count) for {100 * e['same_outcome_frac']:.2f} % of the trajectories
(landed {e['landed']}, escaped {e['escaped']}, still flying at the cap {e['ran_full']}; mean
{e['mean_steps']:.0f} steps); the errors above are over those.

## Density, {d['particles']:.3g} particles, same Philox streams

* per-cell density relative L2, FP32 vs FP64: **{d['density_rel_l2']:.3e}**
* relative L2 between two independent FP32 solves (Monte Carlo noise): {d['independent_run_rel_l2']:.3e}
* ratio: {d['ratio_to_noise']:.3f}
* particle-steps: FP64 {d['total_steps']['fp64']}, FP32 {d['total_steps']['fp32']}

## Column density per unit production rate [m^-2 per molecule/s]

| b / R | FP64 | FP32 | FP32/FP64 - 1 | independent FP32 run, rel. diff. |
|---|---|---|---|---|
{rows}
"""


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=float, default=1e8)
    ap.add_argument("--trajectories", type=float, default=1e4)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--md", type=str, default=None)
    ap.add_argument("--agreement", action="store_true")
    args = sys.argv[1:] if argv is None else argv
    a = ap.parse_args(args)
    if a.agreement:
        with Context(a.device) as ctx:
            res = agreement(ctx, int(a.particles) if a.particles != 1e8 else 100_000)
        print(json.dumps(res), flush=True)
        if a.md:
            with open(a.md, "w") as f:
                f.write(agreement_markdown(res, "python -m dsmc_suite_b200.accuracy " + " ".join(args)))
        return
    p = N.params_config(N.RUNNER_BALLISTIC, 470e3, 6.26e10, 50, 20261203)
    surf = W.config_surface()
    with Context(a.device) as ctx:
        res = {"endpoint": endpoint_errors(ctx, p, surf, int(a.trajectories), a.steps),
               "density": density_errors(ctx, p, surf, int(a.particles))}
    print(json.dumps(res), flush=True)
    if a.md:
        with open(a.md, "w") as f:
            f.write(markdown(res, "python -m dsmc_suite_b200.accuracy " + " ".join(args)))


if __name__ == "__main__":
    main()
