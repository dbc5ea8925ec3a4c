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
        pid0, n = shard.particle_range(rank, world, N_PER_RANK)
        r = O.run(p, S, n, pid_begin=pid0, nthreads=2, particles=False)
        den, hor = shard.allreduce_grids(dist, r["density"], r["horizon"])
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


def test_shard_ranges():
    from dsmc_suite_b200 import shard
    assert [shard.particle_range(r, 4, 10) for r in range(4)] == [(0, 10), (10, 10), (20, 10), (30, 10)]
    parts = [shard.split_range(r, 3, 10) for r in range(3)]
    assert parts == [(0, 4), (4, 3), (7, 3)]
    with pytest.raises(ValueError):
        shard.particle_range(2, 2, 5)
