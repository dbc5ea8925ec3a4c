"""The multi-rank path on CPU: two gloo ranks (separate processes on 127.0.0.1) each solve their
particle-id shard with the oracle (Philox streams, fixed-point grids) and sum the grids with one
all-reduce; the result equals one process solving every id, bit for bit. This is the same
sharding and reduction bench.py runs over NCCL with the CUDA path on each GPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

N_PER_RANK = 150


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_phase1(rank, world, port, out_dir):
    """Phase 1 of the collisional two-phase solve on one rank: its id shard with per-cell speed
    histograms, then one all-reduce of density, horizon and histograms together (the histograms
    feed the FP64 CDF fits, which every rank then computes from the same reduced counts)."""
    import sys
    from datetime import timedelta
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    from dsmc_suite_b200 import _native as N, shard
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        p = N.params_config(N.RUNNER_BALLISTIC)
        p.n_speed_bins = 64
        ico = N.Icosphere(3)
        S = N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())
        pid0, n = shard.particle_range(rank, world, N_PER_RANK)
        r = O.run(p, S, n, pid_begin=pid0, nthreads=2, particles=False, speed_hist=True)
        den, hor, hist = shard.allreduce_grids(dist, r["density"], r["horizon"], r["speed_hist"])
        np.savez(os.path.join(out_dir, f"phase1_{rank}.npz"), density=den, horizon=hor, hist=hist)
    finally:
        dist.destroy_process_group()


def _rank_wrap(rank, world, port, out_dir):
    """Words above 2^63 travel as negative int64: the reduced words must still be the uint64 sums
    modulo 2^64, in the original shapes."""
    import sys
    from datetime import timedelta
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    from dsmc_suite_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        a = np.array([[2**63 + 5, 7], [2**64 - 1, 0]], dtype=np.uint64) + np.uint64(rank)
        b = np.arange(5, dtype=np.uint64) * np.uint64(rank + 1)
        ra, rb = shard.allreduce_grids(dist, a, b)
        np.savez(os.path.join(out_dir, f"wrap_{rank}.npz"), a=ra, b=rb)
    finally:
        dist.destroy_process_group()


def _rank_main(rank, world, port, model, out_dir):
    import sys
    from datetime import timedelta
    from pathlib import Path
    root = str(Path(__file__).resolve().parents[1])
    sys.path.insert(0, root)
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import torch.distributed as dist
    from dsmc_suite_b200 import _native as N, shard
    from oracle import oracle as O
    from conftest import cold_T
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        if model == "reference":
            p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
            S = N.SurfaceInputs(T_map=cold_T(N))
        else:
            p = N.params_config(N.RUNNER_BALLISTIC)
            ico = N.Icosphere(3)
            S = N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())
        def solve_range(pid0, n):
            r = O.run(p, S, n, pid_begin=pid0, nthreads=2, particles=False)
            return r["density"], r["horizon"]

        den, hor = shard.sharded_solve(dist, solve_range, N_PER_RANK)
        if rank == 0:
            np.savez(os.path.join(out_dir, "reduced.npz"), density=den, horizon=hor)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("model", ["config", "reference"])
def test_two_rank_shards_reduce_to_the_one_process_result(N, O, tmp_path, model):
    import multiprocessing as mp
    from conftest import cold_T
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, model, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    red = np.load(tmp_path / "reduced.npz")
    if model == "reference":
        p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
        S = N.SurfaceInputs(T_map=cold_T(N))
    else:
        p = N.params_config(N.RUNNER_BALLISTIC)
        ico = N.Icosphere(3)
        S = N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())
    whole = O.run(p, S, world * N_PER_RANK, nthreads=2, particles=False)
    np.testing.assert_array_equal(red["density"], np.asarray(whole["density"]).reshape(red["density"].shape))
    np.testing.assert_array_equal(red["horizon"], np.asarray(whole["horizon"]).reshape(red["horizon"].shape))
    assert red["density"].any()


def test_two_rank_phase1_histograms_reduce_to_the_one_process_result(N, O, tmp_path):
    """Phase 1 sharded over two gloo ranks: after one all-reduce every rank holds the density,
    horizon and per-cell speed histograms of one process solving all ids, bit for bit, so the
    replicated FP64 fits of phase 2 start from identical counts on every rank."""
    import multiprocessing as mp
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_phase1, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    p = N.params_config(N.RUNNER_BALLISTIC)
    p.n_speed_bins = 64
    ico = N.Icosphere(3)
    S = N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())
    whole = O.run(p, S, world * N_PER_RANK, nthreads=2, particles=False, speed_hist=True)
    for r in range(world):
        red = np.load(tmp_path / f"phase1_{r}.npz")
        np.testing.assert_array_equal(red["hist"], np.asarray(whole["speed_hist"]).reshape(red["hist"].shape))
        np.testing.assert_array_equal(red["density"], np.asarray(whole["density"]).reshape(red["density"].shape))
        np.testing.assert_array_equal(red["horizon"], np.asarray(whole["horizon"]).reshape(red["horizon"].shape))
    assert red["hist"].sum() > 0


def _phase2_inputs(N, O, p1, hist, density, n1):
    """Phase-2 collision inputs from phase-1 results: the oracle's FP64 degree-6 fit of every
    cell with more than 8 counts, the background from the weighted residence times. Every rank
    calls it on the same reduced counts, so every rank holds the same tables."""
    import ctypes as C
    from dsmc_suite_b200 import workloads as W
    ncell = p1.ncell
    coef, box = np.zeros((ncell, N.CDF_STRIDE)), np.zeros((ncell, 4))
    total, valid = np.zeros(ncell), np.zeros(ncell, dtype=np.int32)
    L = O.lib()
    for k in np.nonzero(hist.sum(axis=1) > 8)[0]:
        h = np.ascontiguousarray(hist[k])
        valid[k] = L.or_fit_cell_from_hist(h.ctypes.data_as(C.POINTER(C.c_uint64)), p1.n_speed_bins,
                                           p1.speed_bin_width, 6, O._p(coef[k]), O._p(box[k]),
                                           O._p(total[k:k + 1]))
    nden = W.number_density(p1, density, n1, W.PRODUCTION_RATE)
    col = N.CollisionInputs(nden.ravel(), W.fit_layout(p1, coef), W.fit_layout(p1, box),
                            W.fit_layout(p1, total[:, None]).ravel(),
                            W.fit_layout(p1, valid[:, None]).ravel(), 6)
    p2 = N.params_config(N.RUNNER_ADVANCED)
    p2.seed = p1.seed + 1
    return p2, col


def _two_phase_setup(N):
    p1 = N.params_config(N.RUNNER_BALLISTIC)
    p1.n_speed_bins = 64
    ico = N.Icosphere(3)
    return p1, N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())


def _rank_two_phase(rank, world, port, out_dir):
    """Both phases of the collisional solve sharded by particle id: phase 1 on the rank's ids, one
    all-reduce of density, horizon and histograms; the replicated fits; phase 2 on the rank's ids
    against the fitted tables, one all-reduce of its grids."""
    import sys
    from datetime import timedelta
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    from dsmc_suite_b200 import _native as N, shard
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        p1, S = _two_phase_setup(N)
        pid0, n = shard.particle_range(rank, world, N_PER_RANK)
        r1 = O.run(p1, S, n, pid_begin=pid0, nthreads=2, particles=False, speed_hist=True)
        den1, _, hist = shard.allreduce_grids(dist, r1["density"], r1["horizon"], r1["speed_hist"])
        p2, col = _phase2_inputs(N, O, p1, hist, den1, world * N_PER_RANK)
        r2 = O.run(p2, S, n, collision=col, pid_begin=pid0, nthreads=2, particles=False)
        den2, hor2 = shard.allreduce_grids(dist, r2["density"], r2["horizon"])
        ncol = shard.allreduce_grids(dist, np.array([r2["n_collisions"]], dtype=np.uint64))[0]
        np.savez(os.path.join(out_dir, f"phase2_{rank}.npz"), density=den2, horizon=hor2,
                 valid=col.valid, coef=col.coef, ncol=ncol)
    finally:
        dist.destroy_process_group()


def test_two_rank_two_phase_solve_reduces_to_the_one_process_result(N, O, tmp_path):
    """The collisional two-phase solve over two gloo ranks: the fits every rank replicates from the
    reduced phase-1 counts are identical, and the reduced phase-2 grids (with collisions) equal one
    process running both phases over all ids, bit for bit."""
    import multiprocessing as mp
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_two_phase, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    p1, S = _two_phase_setup(N)
    n_all = world * N_PER_RANK
    w1 = O.run(p1, S, n_all, nthreads=2, particles=False, speed_hist=True)
    p2, col = _phase2_inputs(N, O, p1, w1["speed_hist"], w1["density"], n_all)
    w2 = O.run(p2, S, n_all, collision=col, nthreads=2, particles=False)
    assert w2["n_collisions"] > 0
    for r in range(world):
        got = np.load(tmp_path / f"phase2_{r}.npz")
        np.testing.assert_array_equal(got["valid"], col.valid)
        np.testing.assert_array_equal(got["coef"], col.coef)
        np.testing.assert_array_equal(got["density"], np.asarray(w2["density"]).reshape(got["density"].shape))
        np.testing.assert_array_equal(got["horizon"], np.asarray(w2["horizon"]).reshape(got["horizon"].shape))
        assert int(got["ncol"][0]) == w2["n_collisions"]


def test_two_rank_reduction_keeps_uint64_words(tmp_path):
    import multiprocessing as mp
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_wrap, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    a = np.array([[2**63 + 5, 7], [2**64 - 1, 0]], dtype=np.uint64)
    with np.errstate(over="ignore"):
        want_a = a + a + np.uint64(1)           # modulo 2^64
    want_b = np.arange(5, dtype=np.uint64) * np.uint64(3)
    for r in range(world):
        got = np.load(tmp_path / f"wrap_{r}.npz")
        assert got["a"].dtype == np.uint64 and got["a"].shape == (2, 2)
        np.testing.assert_array_equal(got["a"], want_a)
        np.testing.assert_array_equal(got["b"], want_b)


def _rank_strong(rank, world, port, out_dir, n_total):
    """Strong scaling: n_total ids split over the ranks (uneven), through sharded_solve."""
    import sys
    from datetime import timedelta
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    from dsmc_suite_b200 import _native as N, shard
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        p = N.params_config(N.RUNNER_BALLISTIC)
        ico = N.Icosphere(3)
        S = N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())

        def solve_range(pid0, n):
            r = O.run(p, S, n, pid_begin=pid0, nthreads=2, particles=False)
            return r["density"], r["horizon"]

        den, hor = shard.sharded_solve(dist, solve_range, n_total, weak=False)
        np.savez(os.path.join(out_dir, f"strong_{rank}.npz"), density=den, horizon=hor)
    finally:
        dist.destroy_process_group()


def test_two_rank_strong_scaling_split_reduces_to_the_one_process_result(N, O, tmp_path):
    """An odd number of ids split over two ranks (151 + 150): the reduced grids on every rank
    equal one process solving all of them."""
    import multiprocessing as mp
    world, n_total = 2, 301
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_strong, args=(r, world, port, str(tmp_path), n_total))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    p = N.params_config(N.RUNNER_BALLISTIC)
    ico = N.Icosphere(3)
    whole = O.run(p, N.SurfaceInputs(ico=ico, face_T=ico.face_temperature()), n_total, nthreads=2,
                  particles=False)
    for r in range(world):
        got = np.load(tmp_path / f"strong_{r}.npz")
        np.testing.assert_array_equal(got["density"], np.asarray(whole["density"]).reshape(got["density"].shape))
        np.testing.assert_array_equal(got["horizon"], np.asarray(whole["horizon"]).reshape(got["horizon"].shape))


def test_shard_ranges():
    from dsmc_suite_b200 import shard
    assert [shard.particle_range(r, 4, 10) for r in range(4)] == [(0, 10), (10, 10), (20, 10), (30, 10)]
    parts = [shard.split_range(r, 3, 10) for r in range(3)]
    assert parts == [(0, 4), (4, 3), (7, 3)]
    with pytest.raises(ValueError):
        shard.particle_range(2, 2, 5)
