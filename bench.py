#!/usr/bin/env python
"""Benchmark of the test-particle DSMC hot path on B200.

Workload (one "step"): one complete solve of the Ceres-like ballistic problem - 1e8 H2O test
particles per GPU on a Ceres-like body (R 470 km, GM 6.26e10), icosphere surface of 1280 faces with
T = max(110 K, 235 K cos(z)^0.25), flux-weighted Maxwell-Boltzmann launch, Verlet dt 2 s, at most
20,000 steps per particle, photolysis lifetime 2.6e5 s, 50 exponential shells to 10 R x 36 x 72.
Every particle runs to the end of its life; the metric is particle-steps/s (Verlet steps
executed, counted on the device).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One process per GPU (torchrun for N > 1); each rank solves its own 1e8 particles (weak scaling,
disjoint particle ids) and the fixed-point grids are summed across ranks with one NCCL
all-reduce inside the timed step. Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FLOPS_PER_STEP = 60   # algorithmic FP operations of one particle-step (verlet_step + cell +
                      # photolysis + deposit of the reference algorithm)
METRIC = "particle-steps/s"
SEED = 20261203
E2E_CALLS = 3      # timed end-to-end calls of the solve mode (median reported)


def args_parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--particles", type=float, default=1e8, help="particles per GPU per step")
    ap.add_argument("--plain-particles", type=float, default=1e7,
                    help="particles of the plain FP64 comparison solve (rank 0, N=1)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--shape", type=str, default=None,
                    help="launch shape block,blocks_per_sm,steps_per_launch,launches_per_graph")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--solver", choices=["fast32", "fast64"], default="fast32",
                    help="solve: the timed path (FAST_FP32, the default, or the FP64 engine FAST_FP64)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mode", choices=["solve", "batch", "serve", "collisional", "thermal",
                                       "raytrace"], default="solve",
                    help="solve: one Ceres-like ballistic solve per step (default); batch: the "
                         "64-instance batch; serve: the Poisson request stream; collisional: the "
                         "two-phase collisional solve; thermal: the surface thermal model; raytrace: the "
                         "shadow-flux model on a synthetic cratered mesh")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: arrivals per second")
    ap.add_argument("--seconds", type=float, default=60.0, help="serve: arrival window [s]")
    ap.add_argument("--sample", type=float, default=0.05,
                    help="serve: fraction of requests re-solved with the plain FP64 path")
    ap.add_argument("--budget-gb", type=float, default=80.0, help="batch/serve: HBM budget")
    ap.add_argument("--body", choices=sorted(BODY_RG), default="ceres",
                    help="solve: body of the ballistic workload (ceres is the default workload)")
    return ap.parse_args()


# body of the solve-mode workload (--body): the default is the Ceres-like body; the others are
# the Europa- and Moon-like bodies of the 64-instance batch run alone, for profiling their
# relaunch-bound loops
BODY = "ceres"
BODY_RG = {"ceres": (470e3, 6.26e10), "europa": (1561e3, 3.20e12), "moon": (1737e3, 4.90e12)}


def config_problem(N):
    R, GM = BODY_RG[BODY]
    p = N.params_config(N.RUNNER_BALLISTIC, R, GM, 50, SEED)
    ico = N.Icosphere(3)
    S = N.SurfaceInputs(ico=ico, face_T=ico.face_temperature(T_ss=235.0, T_floor=110.0))
    return p, S


CONFIG = {"workload": "ballistic exosphere, 1e8 particles: Ceres-like body, icosphere 1280 faces, "
                      "T=max(110,235cos^0.25), dt 2 s, <=20000 steps, tau 2.6e5 s, "
                      "50 exp shells to 10R x 36 x 72",
          "l2": "flushed before every timed step (256 MiB write)", "seed": SEED}
SOLVER = "FAST_FP32 resident slots, two-sum compensated push"


def workload_config(n: int, world: int) -> dict:
    """The `config` of the solve-mode line: identical in both arms (the GPU arm and the CPU
    reference arm describe the same workload; how each solves it goes in `solver`)."""
    return dict(CONFIG, particles_per_gpu=n, parallelism=f"particle shards x{world}")


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_problem():
    """The bench workload built by the oracle's own set-up (oracle/problems.py), bit-identical to
    config_problem's, so that the CPU legs never load the product library."""
    from oracle import problems as OP
    R, GM = BODY_RG[BODY]
    p = OP.params_config(OP.RUNNER_BALLISTIC, R, GM, 50, SEED)
    ico = OP.Icosphere(3)
    return p, OP.SurfaceInputs(ico=ico, face_T=ico.face_temperature(T_ss=235.0, T_floor=110.0))


def cpu_oracle_rate(seconds: float, nthreads: int, n_hint: int | None = None):
    """The oracle port (plain C, OpenMP over particles, Philox streams) on a bounded sample of
    the same workload. Returns (steps/s, particles, steps, wall seconds)."""
    from oracle import oracle as O
    O.build()
    p, S = oracle_problem()
    if n_hint is None:
        t0 = time.perf_counter()
        r = O.run(p, S, 2000, nthreads=nthreads, particles=False)
        rate = r["total_steps"] / (time.perf_counter() - t0)
        per = r["total_steps"] / 2000
        n_hint = max(2000, int(rate * seconds / per))
    t0 = time.perf_counter()
    r = O.run(p, S, n_hint, pid_begin=10_000_000, nthreads=nthreads, particles=False)
    dt = time.perf_counter() - t0
    return r["total_steps"] / dt, n_hint, r["total_steps"], dt


def cpu_model() -> str:
    """The host CPU's model name (first `model name` of /proc/cpuinfo), or "unknown"."""
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_binary_rate(seconds: float, nthreads: int):
    """The unmodified reference binary (oracle/_ref/dsmc_suite, compiled from the reference's
    own sources) on its own reference-model workload: `dsmc -n N -t cores` on the synthetic
    36 x 72 map. Particle-steps = sum of flight_time / dt of its _ttime.dat (row 4), which
    leaves out escaped particles as the reference records none for them."""
    cli = ROOT / "oracle" / "_ref" / "dsmc_suite"
    if not cli.exists():
        return None
    import tempfile
    from oracle import problems as OP
    T = OP.latlon_temperature(36, 72, T_ss=235.0, T_floor=110.0)
    with tempfile.TemporaryDirectory() as d:
        (Path(d) / "T.dat").write_text("36\n72\n" + "".join(f"{x:.17g}\n" for x in T.ravel()))
        n = 2000
        for _ in range(3):
            t0 = time.perf_counter()
            subprocess.run([str(cli), "dsmc", "-n", str(n), "-t", str(nthreads), "-T",
                            str(Path(d) / "T.dat"), "-o", str(Path(d) / "r")], check=True,
                           capture_output=True)
            dt = time.perf_counter() - t0
            tt = np.array((Path(d) / "r_ttime.dat").read_text().split(), dtype=np.float64)
            steps = float(tt.reshape(5, n)[4].sum() / 5.0)
            if dt > 0.3 * seconds:
                break
            n = int(n * min(20.0, max(1.5, seconds / max(dt, 1e-3))))
    return {"value": steps / dt, "unit": METRIC, "cores": nthreads, "kind": "reference",
            "sample": f"reference binary, its own physics (Ceres R 476.2 km, dt 5 s, 100 "
                      f"uniform shells): dsmc -n {n} -t {nthreads}, {steps:.3e} steps in "
                      f"{dt:.1f} s wall"}


def run_reference_arm(a):
    """The reference arm: the CPU implementation of the path (the oracle port of the reference's
    particle loop, src/dsmc/ballistic.c:97-281, OpenMP over particles on every host core) on the
    solve-mode workload, each step a bounded sample of it. It loads only oracle/ libraries: the
    problem is built by oracle/problems.py. Rank 0 alone runs; other ranks exit at once."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    per_step = max(2.0, 90.0 / max(1, a.steps + a.warmup))
    rate, n, steps, dt = cpu_oracle_rate(per_step, cores)
    for _ in range(a.warmup - 1):
        cpu_oracle_rate(per_step, cores, n)
    rates, secs = [], []
    for _ in range(a.steps):
        r, _, s, d = cpu_oracle_rate(per_step, cores, n)
        rates.append(r)
        secs.append(d)
    value = float(np.sum([r * d for r, d in zip(rates, secs)]) / np.sum(secs))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": float(np.mean(secs) * 1e3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(int(a.particles), a.gpus),
            "solver": "CPU oracle port of the reference algorithm, OpenMP over particles",
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port",
                             "sample": f"{n} particles of the same workload per step (ids from "
                                       f"1e7); the rate is particle-steps over wall time, which "
                                       f"per particle-step is independent of the sample size",
                             "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    refbin = reference_binary_rate(per_step, cores)
    if refbin:
        line["reference_binary"] = refbin
    print(json.dumps(line), flush=True)


def fma_peak(N, device: int, fp64: bool) -> float:
    import ctypes
    from dsmc_suite_b200 import Context
    with Context(device) as c:
        v = ctypes.c_double()
        N.check(N.lib().dsmc_measure_fma_peak(c.h, int(fp64), ctypes.byref(v)), "fma peak", c.h)
        return v.value


def plain_fp64_rate(N, device: int, problems, limit_steps: float = 4e11):
    """Plain FP64 path (one thread per particle, the reference's arithmetic) over the same
    problems, one solve after another, timed with CUDA events on a dedicated stream; stops
    after about limit_steps particle-steps. Returns (steps/s, problems solved)."""
    import torch
    from dsmc_suite_b200 import Context
    stream = torch.cuda.Stream()
    steps, ms, k = 0, 0.0, 0
    with torch.cuda.stream(stream), Context(device) as ctx:
        ctx.set_stream(stream.cuda_stream)
        for P in problems:
            ctx.setup(P.params, P.surface, P.collision)
            ctx.zero()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.run(N.PATH_PLAIN_FP64, 0, P.n)
            e1.record(stream)
            stream.synchronize()
            ms += e0.elapsed_time(e1)
            steps += ctx.stats()["total_steps"]
            k += 1
            if steps >= limit_steps:
                break
    return steps / (ms * 1e-3), k


def fp64_accuracy(N, device: int, items, same_seed_fp64=None):
    """Density error of FP32 results against FP64 solves of the same problems, next to the Monte
    Carlo noise of each: for every (problem, FP32 density) of `items`, rel = |d32 - d64| / |d64|
    with d64 the FAST_FP64 solve on the same Philox streams (or `same_seed_fp64[k]` when given),
    and noise = |d64' - d64| / |d64| with d64' an FP64 solve under another seed. Returns the
    per-problem medians and maxima, the ratio rel / noise, the worst problem, and the relative L2
    of the aggregate grid (all problems' cells together)."""
    from dsmc_suite_b200 import Context
    rels, noises, sizes = [], [], []
    num = den = 0.0
    with Context(device) as ctx:
        for k, (P, d32) in enumerate(items):
            d64 = same_seed_fp64[k] if same_seed_fp64 is not None else \
                ctx.solve(N.PATH_FAST_FP64, P.params, P.surface, P.n, P.collision)["density"]
            q = P.params.copy()
            q.seed = (q.seed + 0x9E3779B97F4A7C15) % 2**64
            d64b = ctx.solve(N.PATH_FAST_FP64, q, P.surface, P.n, P.collision)["density"]
            a, b, c = (np.asarray(x, dtype=np.float64) for x in (d32, d64, d64b))
            nb = float(np.linalg.norm(b))
            rels.append(float(np.linalg.norm(a - b)) / max(nb, 1e-300))
            noises.append(float(np.linalg.norm(c - b)) / max(nb, 1e-300))
            sizes.append(int(P.n))
            num += float(np.sum((a - b) ** 2))
            den += float(np.sum(b * b))
    rels, noises = np.array(rels), np.array(noises)
    ratio = rels / np.maximum(noises, 1e-300)
    w = int(np.argmax(rels))
    return {"problems": len(items), "fp64": "FAST_FP64, same Philox streams",
            "median": float(np.median(rels)), "max": float(rels.max()),
            "aggregate": float(np.sqrt(num / max(den, 1e-300))),
            "noise_median": float(np.median(noises)), "noise_max": float(noises.max()),
            "ratio_to_noise": {"median": float(np.median(ratio)), "max": float(ratio.max())},
            "worst": {"particles": sizes[w], "rel": float(rels[w]), "noise": float(noises[w])},
            "bar": "aggregate <= 1e-3; per problem rel below its own Monte Carlo noise"}


BATCH_CONFIG = {"workload": "batch of 64 ballistic exospheres in one queue; particles "
                            "lognormal median 3e5 sigma_ln 1.17 clipped [1e4, 1e7]; bodies "
                            "Ceres/Europa/Moon; sub-solar T U(100,400) K, longitude uniform; "
                            "20-60 exp shells x 36 x 72; dt 2 s, <=20000 steps",
                "solver": "dsmc_server: FAST_FP32 resident slots, one device work queue, "
                          "rounds replayed as a CUDA graph",
                "l2": "fresh grids every step; 256 MiB L2 flush before each step", "seed": SEED}


def run_batch_mode(a):
    """The 64-instance batch: every step submits the instances and polls until all are fetched.
    value = particle-steps / device time of the rounds (CUDA events); e2e = the same steps /
    wall time of submit (host tables -> device) ... fetch (grids -> host)."""
    import torch
    from dsmc_suite_b200 import _native as N, Server
    from dsmc_suite_b200 import workloads as W
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    torch.cuda.set_device(local)
    probs = W.batch_instances(SEED, 64)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    if a.shape:
        shape = [int(v) for v in a.shape.split(",")]
    else:
        # autotuned on a 5 % copy of the batch (untimed)
        from dsmc_suite_b200 import autotune
        tuned = autotune.tune(probs, local, scale=0.05)
        shape = tuned["shape"]
        BATCH_CONFIG["autotune"] = {"candidates": len(tuned["trials"]), "sample_scale": 0.05,
                                    "best_sample_rate": tuned["rate"],
                                    "worst_sample_rate": min(t["rate"] for t in tuned["trials"])}
    srv = Server(local, hbm_budget=int(a.budget_gb * 1e9), max_requests=4096)
    srv.set_shape(*shape)
    BATCH_CONFIG["launch_shape"] = list(shape)

    last = {}

    def step():
        i0 = srv.info()
        t0 = time.perf_counter()
        tickets = [srv.submit(P.params, P.surface, P.n, P.collision) for P in probs]
        res = srv.run_all()
        last["density"] = [res[t]["density"] for t in tickets]
        wall = time.perf_counter() - t0
        i1 = srv.info()
        steps = sum(r["stats"]["total_steps"] for r in res.values())
        h2d = sum(P.surface.face_T.nbytes + P.surface.ico.face_verts.nbytes +
                  P.surface.ico.split_planes.nbytes + P.surface.ico.base_centroid.nbytes
                  for P in probs)
        d2h = sum(r["density"].nbytes + r["horizon"].nbytes for r in res.values())
        return steps, i1["busy_ms"] - i0["busy_ms"], wall, i1["launches"] - i0["launches"], h2d, d2h

    for _ in range(a.warmup):
        step()
    tot = [0, 0.0, 0.0, 0, 0, 0]
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            r = step()
            tot = [x + y for x, y in zip(tot, r)]
    steps, busy_ms, wall, launches, h2d, d2h = tot
    value = steps / (busy_ms * 1e-3)
    info = srv.info()
    # the same instances grouped by body, one group at a time (device time of its rounds, after
    # the timed steps): high-gravity bodies relaunch every few hundred steps
    per_body = {}
    for body in sorted({P.meta["body"] for P in probs}):
        group = [P for P in probs if P.meta["body"] == body]
        i0 = srv.info()
        for P in group:
            srv.submit(P.params, P.surface, P.n, P.collision)
        res = srv.run_all(grids=False)
        gs = sum(r["stats"]["total_steps"] for r in res.values())
        gms = srv.info()["busy_ms"] - i0["busy_ms"]
        per_body[body] = {"instances": len(group),
                          "steps_per_particle": gs / sum(P.n for P in group),
                          "value": gs / (gms * 1e-3)}
    srv.close()
    accuracy = fp64_accuracy(N, local, list(zip(probs, last["density"])))
    plain, nplain = plain_fp64_rate(N, local, probs)
    peak = fma_peak(N, local, False)
    achieved = value * FLOPS_PER_STEP / 1e12
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": busy_ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": dict(BATCH_CONFIG, instances=len(probs),
                           particles=int(sum(P.n for P in probs))),
            "particle_steps_per_step": steps / a.steps, "gpu_launches": launches,
            "resident_slots": info["slots"], "clocks": clocks.summary(),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": "measured in this run: FP32 FMA-chain kernel",
                         "algorithmic_flops_per_step": FLOPS_PER_STEP},
            "e2e": {"value": steps / wall, "unit": METRIC, "h2d_bytes_per_step": h2d // a.steps,
                    "d2h_bytes_per_step": d2h // a.steps,
                    "api": "dsmc_server_submit/poll/fetch (C ABI, host buffers)",
                    "seconds": wall},
            "plain_fp64": {"value": plain, "unit": METRIC, "instances": nplain,
                           "note": "same instances, solved one after another"},
            "speedup_vs_plain_fp64": value / plain, "per_body": per_body,
            "density_rel_l2_vs_fp64": accuracy}
    print(json.dumps(line), flush=True)


def run_serve_mode(a):
    """The served stream: Poisson arrivals; each request is admitted at the first poll after its arrival
    (or later, when the budget refuses it), and its latency runs from arrival to the poll that
    saw it complete. Throughput = particle-steps of the completed requests / wall time from the
    first arrival to the last completion."""
    import torch
    from dsmc_suite_b200 import _native as N, Context, Server, BudgetExceeded
    from dsmc_suite_b200 import workloads as W
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(local)
    with Context(local) as ctx:
        t_prep = time.perf_counter()
        stream = W.served_stream(ctx, a.rate, a.seconds, SEED)
        t_prep = time.perf_counter() - t_prep
    rng = np.random.default_rng(SEED + 1)
    sample = set(int(i) for i in np.nonzero(rng.uniform(size=len(stream)) < a.sample)[0])
    srv = Server(local, hbm_budget=int(a.budget_gb * 1e9), max_requests=len(stream) + 16)
    if a.shape:
        srv.set_shape(*[int(v) for v in a.shape.split(",")])
    i0 = srv.info()
    backlog: list[int] = []      # indices refused by admission, retried in order
    ticket_of: dict[int, int] = {}
    done: dict[int, dict] = {}
    nxt = 0
    refused = 0
    t0 = srv.now()
    with ClockSampler(local) as clocks:
        while len(done) < len(stream):
            now = srv.now()
            while nxt < len(stream) and t0 + stream[nxt][0] <= now:
                backlog.append(nxt)
                nxt += 1
            while backlog:
                k = backlog[0]
                P = stream[k][1]
                try:
                    ticket_of[srv.submit(P.params, P.surface, P.n, P.collision)] = k
                except BudgetExceeded:
                    refused += 1
                    break
                backlog.pop(0)
            for t in srv.poll():
                k = ticket_of[t]
                r = srv.fetch(t, grids=k in sample)
                r["arrival"] = t0 + stream[k][0]
                done[k] = r
            if srv.info()["active"] == 0 and not backlog and nxt < len(stream):
                time.sleep(max(0.0, min(0.005, t0 + stream[nxt][0] - srv.now())))
    t_end = max(r["t_done"] for r in done.values())
    info = srv.info()
    srv.close()
    lat = np.array([r["t_done"] - r["arrival"] for r in done.values()])
    steps = sum(r["stats"]["total_steps"] for r in done.values())
    wall = t_end - t0
    # density error of the served FP32 results against the plain FP64 path, seeded subsample
    # (the same solves, timed with CUDA events, give the plain FP64 rate on this request mix)
    errs, plain_dens = [], []
    plain_steps, plain_ms = 0, 0.0
    cs = torch.cuda.Stream()
    with torch.cuda.stream(cs), Context(local) as ctx:
        ctx.set_stream(cs.cuda_stream)
        for k in sorted(sample):
            P = stream[k][1]
            ctx.setup(P.params, P.surface, P.collision)
            ctx.zero()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cs)
            ctx.run(N.PATH_PLAIN_FP64, 0, P.n)
            e1.record(cs)
            cs.synchronize()
            plain_ms += e0.elapsed_time(e1)
            plain_steps += ctx.stats()["total_steps"]
            plain_dens.append(ctx.density())
            errs.append(W.rel_l2(done[k]["density"], plain_dens[-1]))
    accuracy = fp64_accuracy(N, local, [(stream[k][1], done[k]["density"]) for k in sorted(sample)],
                             same_seed_fp64=plain_dens) if plain_dens else None
    if accuracy:
        accuracy["fp64"] = "PLAIN_FP64 on the same Philox streams; noise from FAST_FP64 under another seed"
    kinds = [stream[k][1].meta["kind"] for k in range(len(stream))]
    line = {"metric": METRIC, "value": steps / wall, "unit": METRIC, "n_gpus": 1, "steps": 1,
            "warmup": 0, "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": f"served stream: Poisson {a.rate:g} req/s for "
                                   f"{a.seconds:g} s, 70/30 ballistic/collisional, the 64-instance "
                                   f"batch's distributions, own seed per request",
                       "budget_gb": a.budget_gb, "requests": len(stream),
                       "collisional": kinds.count("collisional"), "seed": SEED},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "mean": float(lat.mean()), "max": float(lat.max())},
            "device_busy_frac": (info["busy_ms"] - i0["busy_ms"]) * 1e-3 / wall,
            "gpu_launches": info["launches"] - i0["launches"], "rounds": info["rounds"] - i0["rounds"],
            "admission_refusals": refused, "particles": int(sum(r["n"] for r in done.values())),
            "density_rel_l2_vs_fp64": dict(accuracy or {}, sample=len(errs)),
            "plain_fp64": {"value": plain_steps / (plain_ms * 1e-3) if plain_ms else None,
                           "unit": METRIC, "requests": len(errs),
                           "note": "the subsample's requests solved one after another"},
            "device_rate": steps / ((info["busy_ms"] - i0["busy_ms"]) * 1e-3),
            "prep_seconds": t_prep, "clocks": clocks.summary()}
    if line["plain_fp64"]["value"]:
        line["speedup_vs_plain_fp64"] = line["value"] / line["plain_fp64"]["value"]
    print(json.dumps(line), flush=True)


def run_collisional_mode(a):
    """The two-phase collisional solve: phase 1 (collisionless, per-cell speed histograms) and the degree-6 FP64 fits,
    then each step is one phase-2 solve with hard-sphere collisions (FAST_FP32) timed with CUDA
    events; the plain FP64 path solves the same phase 2 once for the ratio and the density
    relative L2."""
    import torch
    from dsmc_suite_b200 import _native as N, Context, shard
    from dsmc_suite_b200 import workloads as W
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(local)
    n = int(a.particles) if a.particles != 1e8 else 10_000_000
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    ctx = Context(local)
    ctx.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    prob = W.collisional_problem(ctx, "collisional-ceres", 470e3, 6.26e10, 50, SEED, W.sun_vector(0.0),
                                 235.0, n, n)
    t_phase1 = time.perf_counter() - t0
    col, p, S = prob.collision, prob.params, prob.surface
    ctx.setup(p, S, col)
    if a.shape:
        N.check(N.lib().dsmc_set_launch_shape(ctx.h, *[int(v) for v in a.shape.split(",")]),
                "launch shape", ctx.h)

    def solve(path):
        ctx.zero()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record(stream)
        ctx.run(path, 0, n)
        e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1), ctx.stats()

    for _ in range(a.warmup):
        solve(N.PATH_FAST_FP32)
    ms, steps, ncol = 0.0, 0, 0
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            t, st = solve(N.PATH_FAST_FP32)
            ms += t
            steps += st["total_steps"]
            ncol += st["n_collisions"]
    d32 = ctx.density()
    value = steps / (ms * 1e-3)
    t64, st64 = solve(N.PATH_PLAIN_FP64)
    d64 = ctx.density()
    plain = st64["total_steps"] / (t64 * 1e-3)
    ctx.close()
    peak = fma_peak(N, local, False)
    achieved = value * FLOPS_PER_STEP / 1e12
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": "collisional two-phase, 1e7 particles: Ceres-like body, Antoine "
                                   "sublimation-flux source on T=max(110,235cos^0.25), phase 1 "
                                   "collisionless with 64-bin speed histograms per cell, degree-6 "
                                   "FP64 CDF fits, phase 2 hard spheres d=4.6e-10 m, isotropic "
                                   "scattering; production normalised to 2e26 molecules/s "
                                   "(Ceres' observed ~6 kg/s); 50 exp shells x 36 x 72, dt 2 s",
                       "particles": n, "seed": SEED,
                       "l2": "256 MiB flush before each timed solve"},
            "collisions_per_step": ncol / a.steps, "phase1_and_fit_seconds": t_phase1,
            "valid_fits": int(col.valid.sum()), "max_background_m3": prob.meta["max_n_bg"],
            "production_rate_per_s": prob.meta["rate"],
            "clocks": clocks.summary(),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": "measured in this run: FP32 FMA-chain kernel",
                         "algorithmic_flops_per_step": FLOPS_PER_STEP},
            "plain_fp64": {"value": plain, "unit": METRIC, "collisions": st64["n_collisions"]},
            "speedup_vs_plain_fp64": value / plain,
            "density_rel_l2_fp32_vs_fp64": W.rel_l2(d32, d64),
            "independent_run_note": "FP32 and FP64 follow the same Philox streams"}
    print(json.dumps(line), flush=True)


def run_thermal_mode(a):
    """The thermal column model (36 x 72 columns, Ceres defaults): wall time per solve through
    dsmc_thermal_solve_host (host flux and profile set-up, upload, kernel, download), next to the
    reference's own thermal_solve (oracle/_ref, OpenMP on all host cores) when it is built."""
    from dsmc_suite_b200 import _native as N, Context
    from oracle import oracle as O
    tp = N.ThermalParams.default()
    with Context(0) as ctx:
        for _ in range(a.warmup):
            ctx.thermal(36, 72, tp)
        t0 = time.perf_counter()
        kms = 0.0
        for _ in range(a.steps):
            T, h = ctx.thermal(36, 72, tp)
            kms += ctx.last_kernel_ms()
        gpu_s = (time.perf_counter() - t0) / a.steps
    To, _ = O.thermal(36, 72, tp)
    line = {"metric": "thermal solves/s", "value": 1.0 / gpu_s, "unit": "solves/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": gpu_s * 1e3,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"thermal column model, 36 x 72 columns x {h} depth points x "
                                   f"{tp.n_substep} steps, Ceres defaults, analytic flux"},
            "kernel_ms": kms / a.steps,
            "note": "value is end to end through dsmc_thermal_solve_host (host set-up, copies)",
            "max_abs_diff_vs_oracle_K": float(np.abs(T - To).max()),
            "identical_cells_vs_oracle": float(np.mean(T == To))}
    so = ROOT / "oracle" / "_ref" / "libdsmcref.so"
    if so.exists():
        import ctypes
        R = ctypes.CDLL(str(so))
        g = N.SphericalGrid(ftd=36, ffd=72, hd=1, temperature=N.ptr(np.zeros((36, 72))))
        cores = os.cpu_count() or 1
        devnull = os.open(os.devnull, os.O_WRONLY)
        saved = os.dup(1)
        os.dup2(devnull, 1)          # the reference prints progress lines
        try:
            t0 = time.perf_counter()
            R.thermal_solve(ctypes.byref(g), ctypes.byref(tp), None, cores)
            ref_s = time.perf_counter() - t0
        finally:
            os.dup2(saved, 1)
            os.close(devnull)
        line["cpu_baseline"] = {"value": 1.0 / ref_s, "unit": "solves/s", "cores": cores,
                                "kind": "reference", "sample": "one full solve, reference build"}
    print(json.dumps(line), flush=True)


def run_raytrace_mode(a):
    """The shadow-flux model on a synthetic cratered icosphere (81,920 faces, 24 phases, 50
    samples per face): shadow rays per second through dsmc_shadow_flux_host, BVH build and
    transfers included."""
    from dsmc_suite_b200 import _native as N, Context
    from dsmc_suite_b200 import workloads as W
    spot, facet = W.cratered_mesh(6, craters=64, depth=0.2, width=0.12)
    n = N.mesh_normals(spot, facet)["normal"]
    tt, nm, za = 24, 50, 12.3 / 180 * np.pi
    with Context(0) as ctx:
        for _ in range(a.warmup):
            F = ctx.shadow_flux(spot, facet, n, za, tt, nm)
        t0 = time.perf_counter()
        kms = 0.0
        for _ in range(a.steps):
            F = ctx.shadow_flux(spot, facet, n, za, tt, nm)
            kms += ctx.last_kernel_ms()
        dt = (time.perf_counter() - t0) / a.steps
        kms /= a.steps
    phi = ((np.arange(tt) + 0.5) / tt) * 2.0 * np.pi + np.pi
    sun = np.stack([np.cos(-za) * np.sin(phi), np.cos(-za) * np.cos(phi), np.full(tt, np.sin(-za))], 1)
    rays = int((n @ sun.T >= 0).sum()) * nm
    line = {"metric": "shadow rays/s", "value": rays / dt, "unit": "rays/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": dt * 1e3,
            "higher_is_better": True, "dtype": "fp32 rays, f64 sampling", "data": "synthetic",
            "config": {"workload": f"cratered icosphere, {len(facet)} faces, {tt} phases x {nm} "
                                   f"samples, {rays} rays per solve"},
            "kernel_ms": kms, "kernel_rays_per_s": rays / (kms * 1e-3) if kms else None,
            "note": "value is end to end through dsmc_shadow_flux_host (BVH build, copies)",
            "shadowed_fraction": float(1.0 - F.sum() / np.clip(n @ sun.T, 0, None).sum()),
            "cpu_baseline": None,
            "cpu_baseline_note": "the reference traces with Intel Embree, not installed here"}
    print(json.dumps(line), flush=True)


def main():
    global BODY
    a = args_parse()
    BODY = a.body
    if BODY != "ceres":
        R, GM = BODY_RG[BODY]
        CONFIG["workload"] = (f"ballistic exosphere, 1e8 particles, {BODY}-like body (R {R / 1e3:g} km, GM "
                              f"{GM:g}): icosphere 1280 faces, T=max(110,235cos^0.25), dt 2 s, "
                              f"<=20000 steps, tau 2.6e5 s, 50 exp shells to 10R x 36 x 72")
    if a.impl == "reference":
        return run_reference_arm(a)
    if a.mode == "thermal":
        return run_thermal_mode(a)
    if a.mode == "raytrace":
        return run_raytrace_mode(a)
    if a.mode == "collisional":
        return run_collisional_mode(a)
    if a.mode == "batch":
        return run_batch_mode(a)
    if a.mode == "serve":
        return run_serve_mode(a)
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from dsmc_suite_b200 import _native as N, Context, shard

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    # One dedicated stream for the library's kernels, the L2 flush and the timing events (the
    # legacy default stream has handle 0, which the C ABI reads as "the context's own stream").
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = Context(local)
    ctx.set_stream(stream.cuda_stream)
    p, S = config_problem(N)
    n = int(a.particles)
    pid0, _ = shard.particle_range(rank, world, n)   # weak scaling: disjoint id shards
    ctx.setup(p, S)
    if a.shape:
        shape = [int(v) for v in a.shape.split(",")]
        N.check(N.lib().dsmc_set_launch_shape(ctx.h, *shape), "launch shape", ctx.h)
        CONFIG["launch_shape"] = shape
    ncell, nh = p.ncell, p.ftd * p.ffd
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    red = torch.zeros(ncell + nh, dtype=torch.int64, device="cuda") if world > 1 else None
    L = N.lib()

    timed_path = N.PATH_FAST_FP64 if a.solver == "fast64" else N.PATH_FAST_FP32

    def solve_step():
        ctx.zero()
        ctx.run(timed_path, pid0, n)
        if red is not None:
            d_ptr = red.data_ptr()
            N.check(L.dsmc_copy_grids_device(ctx.h, C_u64(d_ptr), C_u64(d_ptr + 8 * ncell)), "copy", ctx.h)
            shard.allreduce_buffer(dist, red)

    import ctypes
    def C_u64(addr):
        return ctypes.cast(ctypes.c_void_p(addr), ctypes.POINTER(ctypes.c_uint64))

    for _ in range(a.warmup):
        solve_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    steps_done, launches = 0, 0
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        for k in range(a.steps):
            flush.zero_()
            ev[k][0].record(stream)
            solve_step()
            ev[k][1].record(stream)
            st = ctx.stats()
            steps_done += st["total_steps"]
            li = (ctypes.c_int64(), ctypes.c_int64())
            L.dsmc_get_launch_info(ctx.h, ctypes.byref(li[0]), ctypes.byref(li[1]))
            launches += li[0].value
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    t_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    nslots = li[1].value
    tot = torch.tensor([t_ms, float(steps_done)], dtype=torch.float64, device="cuda")
    if world > 1:
        t_max = tot[:1].clone()
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        s_sum = tot[1:].clone()
        dist.all_reduce(s_sum, op=dist.ReduceOp.SUM)
        t_ms, steps_all = float(t_max.item()), float(s_sum.item())
    else:
        steps_all = float(steps_done)
    value = steps_all / (t_ms * 1e-3)
    per_rank_rate = steps_done / (t_ms * 1e-3)

    # roofline of the push kernel: algorithmic FP ops / time against the measured FP32 FMA peak
    fp64_timed = a.solver == "fast64"
    peak = ctypes.c_double()
    N.check(L.dsmc_measure_fma_peak(ctx.h, 1 if fp64_timed else 0, ctypes.byref(peak)), "fma peak", ctx.h)
    achieved = per_rank_rate * FLOPS_PER_STEP / 1e12
    traffic = None
    prof = ROOT / "profiles" / "fast_kernel_traffic.json"
    if prof.exists() and launches:
        tj = json.loads(prof.read_text())
        # DRAM bytes per particle-step from the ncu capture, scaled to this run's launches
        traffic = tj["dram_bytes_per_step"] * (steps_done / launches)
    roofline = {"bound": "fp64" if fp64_timed else "fp32", "achieved": achieved, "peak": peak.value,
                "unit": "TFLOP/s", "frac": achieved / peak.value if peak.value else None,
                "traffic": None if fp64_timed else traffic,
                "peak_source": f"measured in this run: {'FP64' if fp64_timed else 'FP32'} FMA-chain "
                               "kernel (dsmc_measure_fma_peak)",
                "algorithmic_flops_per_step": FLOPS_PER_STEP}

    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": t_ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if fp64_timed else "fp32",
            "data": "synthetic", "config": workload_config(n, world),
            "solver": "FAST_FP64 resident slots, FP64 push" if fp64_timed else SOLVER,
            "particle_steps_per_step": steps_all / a.steps, "gpu_launches": launches,
            "resident_slots": nslots, "clocks": clocks.summary(), "roofline": roofline}

    if rank == 0 and world == 1:
        d32_last = ctx.density()     # the last timed solve's grid
        # plain FP64 path (one thread per particle, the reference's arithmetic) on the same
        # workload, for the FP32-batched vs plain-FP64 ratio
        npl = int(a.plain_particles)
        ctx.zero()
        ctx.run(N.PATH_PLAIN_FP64, 0, 100000)
        torch.cuda.synchronize()
        ctx.zero()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record(stream)
        ctx.run(N.PATH_PLAIN_FP64, 0, npl)
        e1.record(stream)
        torch.cuda.synchronize()
        pst = ctx.stats()["total_steps"]
        plain = pst / (e0.elapsed_time(e1) * 1e-3)
        pk64 = ctypes.c_double()
        N.check(L.dsmc_measure_fma_peak(ctx.h, 1, ctypes.byref(pk64)), "fma peak", ctx.h)
        line["plain_fp64"] = {"value": plain, "unit": METRIC, "particles": npl,
                              "fp64_fma_peak_tflops": pk64.value}
        line["speedup_vs_plain_fp64"] = value / plain
    if rank == 0 and world == 1 and not fp64_timed:
        # the FP64 resident-slot engine on the whole workload (same streams): what the FP32
        # compensated push buys over the same engine in FP64, and the FP32 result's error at
        # full size against it
        d32 = d32_last.astype(np.float64)
        ctx.zero()
        ctx.run(N.PATH_FAST_FP64, 0, 100000)   # warm-up: FP64 slots and graphs are set up here
        torch.cuda.synchronize()
        ctx.zero()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record(stream)
        ctx.run(N.PATH_FAST_FP64, pid0, n)
        e1.record(stream)
        torch.cuda.synchronize()
        s64 = ctx.stats()["total_steps"]
        fast64 = s64 / (e0.elapsed_time(e1) * 1e-3)
        d64 = ctx.density().astype(np.float64)
        a64 = fast64 * FLOPS_PER_STEP / 1e12
        line["fast_fp64"] = {"value": fast64, "unit": METRIC, "particles": n,
                             "roofline": {"bound": "fp64", "achieved": a64, "peak": pk64.value,
                                          "unit": "TFLOP/s", "frac": a64 / pk64.value,
                                          "peak_source": "measured in this run: FP64 FMA-chain kernel"},
                             "density_rel_l2_fp32_vs_fp64": float(np.linalg.norm(d32 - d64) / np.linalg.norm(d64))}
        line["speedup_vs_fast_fp64"] = value / fast64

    if not a.no_e2e:
        # end to end through the C ABI with host buffers: surface upload, solve, grid download
        ctx2 = Context(local)
        host = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy()
                for k, v in (("fv", S.ico.face_verts), ("bc", S.ico.base_centroid),
                             ("sp", S.ico.split_planes), ("ft", S.face_T))}
        ico_pinned = N.Icosphere.__new__(N.Icosphere)
        ico_pinned.__dict__.update(S.ico.__dict__)
        ico_pinned.face_verts, ico_pinned.base_centroid, ico_pinned.split_planes = \
            host["fv"], host["bc"], host["sp"]
        S_pin = N.SurfaceInputs(ico=ico_pinned, face_T=host["ft"])
        den_h = torch.zeros(ncell, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        hor_h = torch.zeros(nh, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        stats = N.Stats()
        pe = p.copy()

        def solve_host():
            N.check(L.dsmc_solve_host(ctx2.h, timed_path, ctypes.byref(pe),
                                      ctypes.byref(S_pin.struct), None, n,
                                      N.ptr(den_h, ctypes.c_uint64), N.ptr(hor_h, ctypes.c_uint64),
                                      ctypes.byref(stats)), "solve_host", ctx2.h)

        solve_host()   # warm-up: the context's first call allocates its slots and captures graphs
        # E2E_CALLS timed calls (each: host tables -> device, solve, grids -> host); the median
        # call's wall time and its steps give the rate, the spread is reported beside it
        walls, e2e_counts = [], []
        for _ in range(E2E_CALLS):
            t0 = time.perf_counter()
            solve_host()
            walls.append(time.perf_counter() - t0)
            e2e_counts.append(float(stats.total_steps))
        order = np.argsort(walls)
        mid = int(order[len(order) // 2])
        dt, e2e_steps = walls[mid], e2e_counts[mid]
        if world > 1:
            agg = torch.tensor([dt, e2e_steps], dtype=torch.float64, device="cuda")
            tmax, ssum = agg[:1].clone(), agg[1:].clone()
            dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
            dist.all_reduce(ssum, op=dist.ReduceOp.SUM)
            dt, e2e_steps = float(tmax.item()), float(ssum.item())
        h2d = sum(v.nbytes for v in host.values())
        line["e2e"] = {"value": e2e_steps / dt, "unit": METRIC, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": den_h.nbytes + hor_h.nbytes + ctypes.sizeof(stats),
                       "api": "dsmc_solve_host (C ABI, pinned host buffers)",
                       "seconds": dt, "calls": len(walls),
                       "call_seconds": [round(w, 4) for w in walls],
                       "statistic": "median call"}
        ctx2.close()

    if rank == 0 and world == 1 and not a.no_cpu:
        cores = os.cpu_count() or 1
        rate, ncpu, scpu, dcpu = cpu_oracle_rate(a.cpu_seconds, cores)
        line["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": cores, "kind": "port",
                                "sample": f"{ncpu} particles of the same workload, {scpu} "
                                          f"particle-steps in {dcpu:.1f} s (oracle port, OpenMP)"}
        refbin = reference_binary_rate(a.cpu_seconds, cores)
        if refbin:
            line["cpu_baseline"]["reference_binary"] = refbin
        # one thread, a quarter of the sample time: the per-core rate the OpenMP figure scales
        r1, n1, s1, d1 = cpu_oracle_rate(a.cpu_seconds / 4, 1)
        line["cpu_baseline"]["single_thread"] = {
            "value": r1, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{n1} particles, {s1} particle-steps in {d1:.1f} s"}
        line["cpu_baseline"]["cpu_model"] = cpu_model()

    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
