"""Particle sharding across ranks (one process per GPU).

Test particles are independent - collisions are against the fixed phase-1 background, never
between particles - so a solve of N particles splits into disjoint particle-id ranges, one per
rank, with no exchange until the end. Each rank adds into its own fixed-point grids; one sum
all-reduce of the integer density and horizon grids combines them. Particle streams are keyed by
particle id and the grids are integer sums, so the reduced grids equal a one-GPU solve of all ids
bit for bit (modulo-2^64 sums of the unsigned words, carried as int64). Phase 1 of a collisional
two-phase solve reduces its per-cell speed histograms (uint64 counts) in the same call, and
every rank fits the phase-2 CDF tables from the identical reduced counts.
"""
from __future__ import annotations

import numpy as np


def particle_range(rank: int, world: int, n_per_rank: int) -> tuple[int, int]:
    """(pid_begin, n) of a rank under weak scaling: rank r solves ids [r n, (r + 1) n)."""
    if not (0 <= rank < world) or n_per_rank < 0:
        raise ValueError("rank must lie in [0, world) and n_per_rank >= 0")
    return rank * n_per_rank, n_per_rank


def split_range(rank: int, world: int, n_total: int) -> tuple[int, int]:
    """(pid_begin, n) of a rank under strong scaling: ids [0, n_total) in near-equal parts."""
    if not (0 <= rank < world) or n_total < 0:
        raise ValueError("rank must lie in [0, world) and n_total >= 0")
    base, extra = divmod(n_total, world)
    begin = rank * base + min(rank, extra)
    return begin, base + (1 if rank < extra else 0)


def allreduce_buffer(dist, buf) -> None:
    """The one collective of a sharded solve: an in-place sum all-reduce of an int64 torch tensor
    that holds a rank's fixed-point grids back to back (density, horizon and, in phase 1 of a
    collisional solve, the speed histograms). The unsigned 64-bit words travel as int64, whose
    two's-complement sums are the modulo-2^64 sums of the words. `buf` lives on the rank's GPU
    for NCCL (bench.py fills it with dsmc_copy_grids_device) or on the CPU for gloo."""
    import torch
    if buf.dtype != torch.int64 or not buf.is_contiguous():
        raise ValueError("the grid buffer must be a contiguous int64 tensor")
    dist.all_reduce(buf, op=dist.ReduceOp.SUM)


def allreduce_grids(dist, *grids: np.ndarray, device=None) -> list[np.ndarray]:
    """Sum uint64 host grids over the process group with one allreduce_buffer call. `device` is
    the torch device of the communication buffer ("cuda" for NCCL, None/CPU for gloo)."""
    import torch
    flat = np.concatenate([g.ravel().view(np.int64) for g in grids])
    t = torch.from_numpy(flat.copy())
    if device is not None:
        t = t.to(device)
    allreduce_buffer(dist, t)
    out = t.cpu().numpy().view(np.uint64)
    res, k = [], 0
    for g in grids:
        res.append(out[k:k + g.size].reshape(g.shape).copy())
        k += g.size
    return res


def sharded_solve(dist, solve_range, n: int, weak: bool = True, device=None) -> list[np.ndarray]:
    """One rank's part of a sharded solve: the rank's particle-id range (weak scaling: n ids per
    rank, `particle_range`; strong: n ids in all, `split_range`), solved by
    solve_range(pid_begin, count) -> tuple of uint64 grids (density, horizon, optionally speed
    histograms), then one all-reduce of all of them. Every rank returns the grids of one solve
    of all ids. solve_range may run on the GPU (Context.run + density / horizon) or anywhere
    else; `device` is the communication buffer's torch device ("cuda" for NCCL)."""
    rank, world = dist.get_rank(), dist.get_world_size()
    pid0, count = particle_range(rank, world, n) if weak else split_range(rank, world, n)
    return allreduce_grids(dist, *solve_range(pid0, count), device=device)
