"""Batched and served solves through the dsmc_server_* C ABI (needs a B200).

Bars: a request's density, horizon and statistics are bit-identical
  * to the same problem solved alone by the context's FAST_FP32 path,
  * whether it runs alone or admitted into a queue while other requests are on the GPU, under
    another launch shape;
and admission refuses what does not fit the memory budget or the queue, then admits it once
results have been fetched."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cold_T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def surf(N):
    ico = N.Icosphere(3)
    return N.SurfaceInputs(ico=ico, face_T=ico.face_temperature())


@pytest.fixture(scope="module")
def requests(ctx, N, O, surf):
    """Four problems of different kinds: (name, params, surface, collision, n)."""
    from test_gpu_parity import _config_collision_inputs
    out = []
    pa = N.params_config(N.RUNNER_BALLISTIC)
    pa.seed = 11
    out.append(("config-ballistic", pa, surf, None, 30000))
    pb, col, _ = _config_collision_inputs(ctx, N, O, surf)
    pb.seed = 12
    out.append(("config-collisional", pb, surf, col, 6000))
    pc = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    pc.seed = 13
    out.append(("reference-ballistic", pc, N.SurfaceInputs(T_map=cold_T(N)), None, 5000))
    # Europa-like body, 30 shells, sub-solar point elsewhere, hotter
    ico = surf.ico
    sun = np.array([np.cos(2.0), np.sin(2.0), 0.0])
    pd = N.params_config(N.RUNNER_BALLISTIC, Radii=1561e3, GM=3.20e12, hd=30, seed=14)
    pd.sun[0], pd.sun[1], pd.sun[2] = sun
    sd = N.SurfaceInputs(ico=ico, face_T=ico.face_temperature(sun=sun, T_ss=330.0))
    out.append(("europa-ballistic", pd, sd, None, 20000))
    return out


def _same(a, b):
    np.testing.assert_array_equal(a["density"], b["density"])
    np.testing.assert_array_equal(a["horizon"], b["horizon"])
    assert a["stats"] == b["stats"]


@pytest.fixture(scope="module")
def alone(N, requests):
    from dsmc_suite_b200.server import Server
    res = {}
    with Server(0, hbm_budget=8 * 10**9, max_requests=64) as srv:
        for name, p, s, col, n in requests:
            t = srv.submit(p, s, n, collision=col)
            got = srv.run_all()
            assert list(got) == [t]
            res[name] = got[t]
            assert res[name]["stats"]["n_finished"] == n
    return res


def test_server_matches_context_fast_path(ctx, N, requests, alone):
    for name, p, s, col, n in requests:
        ref = ctx.solve(N.PATH_FAST_FP32, p, s, n, collision=col)
        _same(alone[name], ref)
        assert alone[name]["latency"] >= 0.0


def test_served_results_identical_alone_and_in_mix(N, surf, requests, alone):
    from dsmc_suite_b200.server import Server
    with Server(0, hbm_budget=8 * 10**9, max_requests=64) as srv:
        srv.set_shape(256, 0, 1000, 3)
        filler = N.params_config(N.RUNNER_BALLISTIC, seed=99)
        tickets = {"filler-0": srv.submit(filler, surf, 150000)}
        srv.poll()
        overlapped = 0
        for k, (name, p, s, col, n) in enumerate(requests):
            overlapped += srv.info()["active"] > 0
            tickets[name] = srv.submit(p, s, n, collision=col)
            srv.poll()
            if k == 1:
                f2 = N.params_config(N.RUNNER_BALLISTIC, hd=40, seed=98)
                tickets["filler-1"] = srv.submit(f2, surf, 80000)
        got = srv.run_all()
        info = srv.info()
    assert overlapped == len(requests)      # every request was admitted beside running ones
    assert set(got) == set(tickets.values())
    for name, *_ in requests:
        _same(got[tickets[name]], alone[name])
    assert info["completed"] == info["fetched"] == len(tickets)
    assert info["launches"] >= 3 * info["rounds"] > 0
    assert info["total_steps"] == sum(r["stats"]["total_steps"] for r in got.values())


def test_grouped_admission_changes_no_result(N, requests, alone):
    """Requests admitted between two polls join the queue grouped by hop length (the Europa-like
    request's short hops after the Ceres-like ones): in either submission order every request's
    results are those it has alone."""
    from dsmc_suite_b200.server import Server
    for order in (requests, requests[::-1]):
        with Server(0, hbm_budget=8 * 10**9, max_requests=64) as srv:
            tickets = {name: srv.submit(p, s, n, collision=col) for name, p, s, col, n in order}
            assert srv.info()["active"] == len(order)    # pending until the first poll
            got = srv.run_all()
        for name, *_ in order:
            _same(got[tickets[name]], alone[name])


def test_server_admission_by_budget_and_queue(N, surf):
    from dsmc_suite_b200.server import BudgetExceeded, Server
    p = N.params_config(N.RUNNER_BALLISTIC, seed=5)
    with Server(0, hbm_budget=8 * 10**9, max_requests=4) as probe:
        base = probe.info()["bytes_in_use"]
        probe.submit(p, surf, 1000)
        one = probe.info()["bytes_in_use"] - base
        probe.run_all()
        assert probe.info()["bytes_in_use"] == base     # fetch gave the memory back
    assert one > 129600 * 8
    with Server(0, hbm_budget=base + int(1.5 * one), max_requests=2) as srv:
        t0 = srv.submit(p, surf, 20000)
        with pytest.raises(BudgetExceeded):
            srv.submit(p, surf, 20000)
        assert srv.info()["rejected"] == 1
        first = srv.run_all()
        t1 = srv.submit(p, surf, 20000)        # admitted once the first was fetched
        second = srv.run_all()
        _same(first[t0], second[t1])            # same seed, same particle ids
        # queue capacity: two requests fill it; a third waits until the queue drains
        q = N.params_config(N.RUNNER_BALLISTIC, hd=10, seed=6)
        srv2 = Server(0, hbm_budget=8 * 10**9, max_requests=2)
        try:
            srv2.submit(q, surf, 2000)
            srv2.submit(q, surf, 2000)
            with pytest.raises(BudgetExceeded):
                srv2.submit(q, surf, 2000)
            srv2.run_all()
            srv2.submit(q, surf, 2000)          # the queue restarted from empty
            assert len(srv2.run_all()) == 1
        finally:
            srv2.close()


def test_server_edge_cases(N, surf):
    from dsmc_suite_b200.server import Server
    p = N.params_config(N.RUNNER_BALLISTIC, seed=7)
    with Server(0, hbm_budget=8 * 10**9, max_requests=8) as srv:
        t0 = srv.submit(p, surf, 0)                     # empty request: complete at once
        assert srv.poll() == [t0]
        r = srv.fetch(t0)
        assert r["stats"]["n_finished"] == 0 and not r["density"].any()
        t1 = srv.submit(p, surf, 3000)
        with pytest.raises(N.DsmcError) as e:
            srv.fetch(t1)                               # still running
        assert e.value.status == -5
        srv.run_all()
        with pytest.raises(N.DsmcError):
            srv.fetch(t1)                               # already fetched
        bad = p.copy()
        bad.hd = 0
        with pytest.raises(N.DsmcError):
            srv.submit(bad, surf, 10)
        with pytest.raises(N.DsmcError):
            srv.submit(p, surf, -1)
        assert srv.info()["active"] == 0


def test_autotune_picks_the_fastest_candidate_and_caches_it(N, surf, tmp_path):
    from dsmc_suite_b200 import autotune
    from dsmc_suite_b200.workloads import batch_instances
    probs = batch_instances(seed=5, count=4)
    cands = [(128, 0, 512, 2), (128, 0, 2048, 4)]
    cache = tmp_path / "tune.json"
    r = autotune.tune(probs, 0, scale=0.01, candidates=cands, cache=cache)
    assert tuple(r["shape"]) in cands and len(r["trials"]) == 2
    assert r["rate"] == max(t["rate"] for t in r["trials"]) > 0
    assert autotune.tune(probs, 0, scale=0.01, candidates=cands, cache=cache) == \
        __import__("json").loads(cache.read_text())[next(iter(__import__("json").loads(cache.read_text())))]
