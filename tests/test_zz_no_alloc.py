"""dsmc_solve_fast_noalloc: the FAST_FP32 solve for callers that cannot allocate device memory
(their framework owns every device buffer through its own pool, or their process budgets or
intercepts allocation calls). They hand in device buffers they already hold; the library's
scratch is one fixed device array inside the library.

The test holds its device buffers in torch tensors (the test is the caller here), calls the
entry point through the C ABI twice in a row - a config-model problem, then a reference-model
problem, so stale scratch from the first call would show in the second - and checks each result
against the existing entry point (Context.solve with FAST_FP32). The fast path is deterministic
(every trajectory is a function of its particle id, deposits are integer sums), so the bar is
bit-identical grids and counters. This file is collected last on purpose."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import cold_T

pytestmark = pytest.mark.gpu


def _dev(torch, a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda") if dtype is None else \
        torch.from_numpy(np.ascontiguousarray(a)).to(dtype).to("cuda")


def _dptr(t, ctype=C.c_double):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype))


def _buffers(torch, p):
    """Device buffers the caller owns: density, horizon and the six statistics words (set to a
    non-zero pattern, which the call must clear)."""
    return (torch.zeros(p.ncell, dtype=torch.int64, device="cuda"),
            torch.zeros(p.ftd * p.ffd, dtype=torch.int64, device="cuda"),
            torch.full((6,), 7, dtype=torch.int64, device="cuda"))


def _call(N, p, surf_dev, n, bufs):
    density, horizon, stats = bufs
    rc = N.lib().dsmc_solve_fast_noalloc(C.byref(p), C.byref(surf_dev), 0, n,
                                         _dptr(density, C.c_uint64), _dptr(horizon, C.c_uint64),
                                         _dptr(stats, C.c_uint64), None)
    assert rc == 0, N.lib().dsmc_noalloc_last_error()


def _host(p, bufs):
    density, horizon, stats = bufs
    return (density.cpu().numpy().view(np.uint64).reshape(p.hd, p.ftd, p.ffd),
            horizon.cpu().numpy().view(np.uint64).reshape(p.ftd, p.ffd),
            stats.cpu().numpy())


def _noalloc_solve(N, torch, p, surf_dev, n):
    bufs = _buffers(torch, p)
    _call(N, p, surf_dev, n, bufs)
    torch.cuda.synchronize()
    return _host(p, bufs)


def test_noalloc_matches_existing_entry_point_twice(N, built):
    torch = pytest.importorskip("torch")
    from dsmc_suite_b200 import Context

    # call 1: config model (icosphere surface), device copies of the surface arrays
    ico = N.Icosphere(3)
    fT = ico.face_temperature()
    keep = [_dev(torch, ico.face_verts), _dev(torch, fT), _dev(torch, ico.base_centroid),
            _dev(torch, ico.split_planes)]
    sd = N.Surface()
    sd.nface, sd.nlevel = ico.nface, ico.nlevel
    sd.face_verts, sd.face_T, sd.base_centroid, sd.split_planes = (_dptr(t) for t in keep)
    pc = N.params_config(N.RUNNER_BALLISTIC)
    n1 = 40000
    d1, h1, s1 = _noalloc_solve(N, torch, pc, sd, n1)

    # call 2: reference model (latitude-longitude map with cold regions)
    T = cold_T(N)
    Td = _dev(torch, T)
    sr = N.Surface()
    sr.T_map = _dptr(Td)
    pr = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    n2 = 30000
    d2, h2, s2 = _noalloc_solve(N, torch, pr, sr, n2)

    with Context(0) as ctx:
        ref1 = ctx.solve(N.PATH_FAST_FP32, pc, N.SurfaceInputs(ico=ico, face_T=fT), n1)
        ref2 = ctx.solve(N.PATH_FAST_FP32, pr, N.SurfaceInputs(T_map=T), n2)
    for (d, h, s), ref, n in (((d1, h1, s1), ref1, n1), ((d2, h2, s2), ref2, n2)):
        np.testing.assert_array_equal(d, ref["density"])
        np.testing.assert_array_equal(h, ref["horizon"])
        st = ref["stats"]
        assert int(s[0]) == st["total_steps"] > 0
        assert int(s[1]) == st["n_escaped"] and int(s[4]) == st["n_finished"] == n

    # A third call allocates no device memory: the device's free memory is the same before and
    # after it (its buffers are the caller's, allocated beforehand).
    bufs = _buffers(torch, pc)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _call(N, pc, sd, n1, bufs)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "the no-allocation call allocated device memory"
    d3, h3, _ = _host(pc, bufs)
    np.testing.assert_array_equal(d3, ref1["density"])
    np.testing.assert_array_equal(h3, ref1["horizon"])


def test_noalloc_long_lived_particles(N, built):
    """A few reference-model particles that live for 9e6 steps each (no photolysis, no escape by
    launch speed, a 9e6-step life cap): the tail of the solve runs more than a thousand launches
    in which no particle finishes, which must not read as a stalled queue; the result equals the
    existing entry point's."""
    torch = pytest.importorskip("torch")
    from dsmc_suite_b200 import Context
    p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    p.ve, p.lifetime, p.wdecay, p.w_min = 1e30, 1e30, 1.0, -1.0
    p.life_step_cap = 9_000_000
    T = N.latlon_temperature(36, 72, T_ss=235.0, T_floor=110.0)
    Td = _dev(torch, T)
    sr = N.Surface()
    sr.T_map = _dptr(Td)
    n = 8
    d, h, s = _noalloc_solve(N, torch, p, sr, n)
    with Context(0) as ctx:
        ref = ctx.solve(N.PATH_FAST_FP32, p, N.SurfaceInputs(T_map=T), n)
    np.testing.assert_array_equal(d, ref["density"])
    np.testing.assert_array_equal(h, ref["horizon"])
    assert int(s[0]) == ref["stats"]["total_steps"] and int(s[4]) == n
    assert int(s[0]) > 9_000_000, "no particle reached the life cap"


def test_noalloc_rejects_sizes_beyond_its_scratch(N, built):
    pytest.importorskip("torch")
    p = N.params_config(N.RUNNER_BALLISTIC, hd=4000)
    s = N.Surface()
    dummy = C.cast(C.c_void_p(16), C.POINTER(C.c_uint64))
    rc = N.lib().dsmc_solve_fast_noalloc(C.byref(p), C.byref(s), 0, 10, dummy, dummy, dummy, None)
    assert rc == -1
    assert b"too large" in N.lib().dsmc_noalloc_last_error()
    p2 = N.params_config(N.RUNNER_BALLISTIC)
    p2.model = 5
    assert N.lib().dsmc_solve_fast_noalloc(C.byref(p2), C.byref(s), 0, 10, dummy, dummy, dummy, None) == -1
    assert b"unknown physics model" in N.lib().dsmc_noalloc_last_error()
    p3 = N.params_config(N.RUNNER_BALLISTIC)
    for pid0, n in ((2**32 - 5, 10), (2**62, 2**62), (0, 2**32 + 1)):
        assert N.lib().dsmc_solve_fast_noalloc(C.byref(p3), C.byref(s), pid0, n, dummy, dummy, dummy,
                                               None) == -1
        assert b"[0, 2^32)" in N.lib().dsmc_noalloc_last_error()
