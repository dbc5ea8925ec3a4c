"""Launch-shape autotuner of the FAST_FP32 engine (batched and served solves).

The engine's throughput depends on the launch shape - threads per block, resident blocks per SM,
Verlet steps per slot per launch (K) and launches per captured graph (G) - and on the workload
(how often particles relaunch, how long they live, how many instances share the queue). The
tuner solves a scaled-down copy of the caller's problems (every particle count times `scale`,
same bodies, grids and seeds) under each candidate shape through a Server, times the rounds with
the server's CUDA events, and returns the fastest shape. Results do not depend on the shape, so
the choice affects speed only. Choices are cached per GPU name and workload signature in a JSON
file when a cache path is given.

There is no deposit tile to tune: deposits accumulate per particle in registers for the current
cell and are flushed with one 64-bit atomic when the particle leaves it.
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

from .server import Server

# (block, blocks_per_sm, steps_per_launch, launches_per_graph)
CANDIDATES = [(b, bps, k, g) for b, bps in ((128, 3), (128, 4), (128, 5), (256, 2))
              for k in (1024, 2048, 4096) for g in (2, 4, 8)]


def signature(problems) -> str:
    h = hashlib.sha1()
    for P in problems:
        p = P.params
        h.update(bytes(p))
        h.update(str(P.n).encode())
        h.update(b"c" if P.collision is not None else b"b")
    return h.hexdigest()[:16]


def tune(problems, device: int = 0, scale: float = 0.05, candidates=None, min_particles: int = 1000,
         cache: str | Path | None = None, budget: int = 40 * 10**9) -> dict:
    """Fastest launch shape for `problems` (objects with params, surface, n, collision).
    Returns {"shape": (block, blocks_per_sm, K, G), "rate": steps/s, "trials": [...]}."""
    import torch
    cands = list(candidates or CANDIDATES)
    key = f"{torch.cuda.get_device_name(device)}|{signature(problems)}|{scale}|{cands}"
    if cache is not None and Path(cache).exists():
        known = json.loads(Path(cache).read_text())
        if key in known:
            return known[key]
    trials = []
    with Server(device, hbm_budget=budget, max_requests=max(64, 2 * len(problems))) as srv:
        for shape in cands:
            srv.set_shape(*shape)
            i0 = srv.info()
            for P in problems:
                srv.submit(P.params, P.surface, max(min_particles, int(P.n * scale)), P.collision)
            res = srv.run_all(grids=False)
            i1 = srv.info()
            steps = sum(r["stats"]["total_steps"] for r in res.values())
            ms = i1["busy_ms"] - i0["busy_ms"]
            trials.append({"shape": list(shape), "rate": steps / (ms * 1e-3), "ms": ms})
    best = max(trials, key=lambda t: t["rate"])
    out = {"shape": best["shape"], "rate": best["rate"], "scale": scale, "trials": trials}
    if cache is not None:
        known = json.loads(Path(cache).read_text()) if Path(cache).exists() else {}
        known[key] = out
        Path(cache).write_text(json.dumps(known, indent=1))
    return out
