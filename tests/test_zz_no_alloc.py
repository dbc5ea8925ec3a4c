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


def _noalloc_solve(N, torch, p, surf_dev, n):
    ncell, nh = p.ncell, p.ftd * p.ffd
    density = torch.zeros(ncell, dtype=torch.int64, device="cuda")
    horizon = torch.zeros(nh, dtype=torch.int64, device="cuda")
    stats = torch.full((6,), 7, dtype=torch.int64, device="cuda")   # the call must zero these
    rc = N.lib().dsmc_solve_fast_noalloc(C.byref(p), C.byref(surf_dev), 0, n,
                                         _dptr(density, C.c_uint64), _dptr(horizon, C.c_uint64),
                                         _dptr(stats, C.c_uint64), None)
    assert rc == 0, N.lib().dsmc_noalloc_last_error()
    torch.cuda.synchronize()
    return (density.cpu().numpy().view(np.uint64).reshape(p.hd, p.ftd, p.ffd),
            horizon.cpu().numpy().view(np.uint64).reshape(p.ftd, p.ffd),
            stats.cpu().numpy())


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


def test_noalloc_rejects_sizes_beyond_its_scratch(N, built):
    pytest.importorskip("torch")
    p = N.params_config(N.RUNNER_BALLISTIC, hd=4000)
    s = N.Surface()
    dummy = C.cast(C.c_void_p(16), C.POINTER(C.c_uint64))
    rc = N.lib().dsmc_solve_fast_noalloc(C.byref(p), C.byref(s), 0, 10, dummy, dummy, dummy, None)
    assert rc == -1
    assert b"too large" in N.lib().dsmc_noalloc_last_error()
