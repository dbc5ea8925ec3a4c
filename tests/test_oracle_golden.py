"""The CPU oracle against the reference's own known answers and golden vectors.

The fixtures in tests/golden/ were produced by the reference compiled from its own sources
(tests/golden/make_golden.py). In rand_r mode with one thread the oracle must reproduce the
reference's `-t 1` runs file for file, and its scalar functions bit for bit."""
from __future__ import annotations

import ctypes as C
import hashlib
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, cold_T


def test_philox_known_answers(O):
    # Known-answer vectors of Philox4x32-10 (Salmon et al., SC'11, Random123 distribution).
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E,
                                                            0xA20BC7C6, 0x6D5451FD]
    assert O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                    [0xA4093822, 0x299F31D0]) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_verlet_kat_circular_orbit(O, golden):
    """tests/test_verlet.c:12-56: circular orbit at 2R, h = 1 s, 1000 steps."""
    L = O.lib()
    G, M, R = 6.67e-11, 9.39e20, 476.2e3
    GM = G * M
    r0 = 2.0 * R
    s = np.array([r0, 0.0, 0.0])
    v = np.array([0.0, np.sqrt(G * M / r0), 0.0])
    oa = np.array([G * M * s[0] / (r0 * r0 * r0), 0.0, 0.0])
    E0 = 0.5 * (v @ v) - G * M / np.sqrt(s @ s)
    for _ in range(1000):
        L.or_verlet_step(O._p(s), O._p(v), O._p(oa), GM, 1.0, R, 10 * R, None)
    E1 = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - G * M / np.sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2])
    kat = golden["meta"]["test_verlet"]
    assert f"{E0:.10e}" == f"{kat['E0']:.10e}"
    assert f"{E1:.10e}" == f"{kat['E1']:.10e}"
    assert abs(E1 - E0) / abs(E0) < 1e-3


def test_velocity_table_kat(O, golden):
    """tests/test_verlet.c:59-96: every row non-empty; mean of 10,000 samples at 200 K with
    seed 42 is 100.0 m/s (the table saturates at 1000 entries of the lowest speeds)."""
    vt = O.vtable()
    assert min(vt.count) > 0
    np.testing.assert_array_equal(np.array(vt.speeds), golden["scalars"]["vt_speeds"])
    np.testing.assert_array_equal(np.array(vt.count), golden["scalars"]["vt_count"])
    libc = C.CDLL(None)
    libc.rand_r.restype = C.c_int
    seed = C.c_uint(42)
    s = 0.0
    for _ in range(10000):
        s += O.lib().or_velocity_sample_word(C.byref(vt), 200.0, libc.rand_r(C.byref(seed)))
    assert f"{s / 10000:.1f}" == f"{golden['meta']['test_verlet']['mean_v_200K']:.1f}" == "100.0"


def test_velocity_sample_sequences(O, golden):
    vt = O.vtable()
    libc = C.CDLL(None)
    libc.rand_r.restype = C.c_int
    g = golden["scalars"]
    for T, ref in zip(g["vs_T"], g["vs_values"]):
        seed = C.c_uint(42)
        got = [O.lib().or_velocity_sample_word(C.byref(vt), float(T), libc.rand_r(C.byref(seed)))
               for _ in range(len(ref))]
        np.testing.assert_array_equal(got, ref)


def test_polyfit_kat(O, golden):
    """tests/test_verlet.c:99-135: exact cubic on x = 0..10 gives (2, -1, 3, -1)."""
    x = np.arange(11.0)
    y = 2 * x ** 3 - x ** 2 + 3 * x - 1
    c = np.zeros(7)
    assert O.lib().or_polyfit(O._p(x), O._p(y), 11, 3, O._p(c)) == 0
    assert [round(v, 4) for v in c[:4]] == golden["meta"]["test_verlet"]["coefficients"]
    val = ((c[0] * 5 + c[1]) * 5 + c[2]) * 5 + c[3]
    assert abs(val - 239.0) < 0.01


def test_polyfit_matches_reference(O, golden):
    g = golden["scalars"]
    for deg, (x, y, cref) in enumerate(zip(g["polyfit_x"], g["polyfit_y"], g["polyfit_c"]), 1):
        c = np.zeros(7)
        assert O.lib().or_polyfit(O._p(np.ascontiguousarray(x)), O._p(np.ascontiguousarray(y)),
                                  len(x), deg, O._p(c)) == 0
        np.testing.assert_array_equal(c[:deg + 1], cref[:deg + 1])


def test_verlet_matches_reference_bit_for_bit(O, golden):
    g = golden["scalars"]
    L = O.lib()
    for i in range(len(g["verlet_s0"])):
        s = g["verlet_s0"][i].copy()
        v = g["verlet_v0"][i].copy()
        R = np.sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2])
        oa = np.array([g["verlet_GM"] * s[k] / (R * R * R) for k in range(3)])
        ds = C.c_double()
        st, k = 0, 0
        while k < g["verlet_steps"] and st == 0:
            st = L.or_verlet_step(O._p(s), O._p(v), O._p(oa), float(g["verlet_GM"]),
                                  float(g["verlet_h"]), float(g["verlet_Radii"]),
                                  float(g["verlet_max_height"]), C.byref(ds))
            k += 1
        assert st == g["verlet_status"][i] and k == g["verlet_taken"][i]
        np.testing.assert_array_equal(s, g["verlet_s"][i])
        np.testing.assert_array_equal(v, g["verlet_v"][i])
        np.testing.assert_array_equal(oa, g["verlet_oa"][i])
        assert ds.value == g["verlet_ds"][i]


def test_grid_index_functions(O, golden):
    g = golden["scalars"]
    td, fd = C.c_int(), C.c_int()
    for a, b, ref in zip(g["index_thi"], g["index_fi"], g["index_td_fd"]):
        O.lib().or_spherical_to_index(float(a), float(b), 36, 72, C.byref(td), C.byref(fd))
        assert (td.value, fd.value) == tuple(ref)
    R, a2 = 476.2e3, 0.04
    import math
    for r, ref in zip(g["expht_radii"], g["expht_index"]):
        assert O.lib().or_exp_ht_index(float(r), R, float(g["expht_unih"]), a2,
                                       math.log(1.0 + a2)) == ref


def test_cdf_sample_matches_reference(O, golden):
    g = golden["scalars"]
    for fit, u, nn, vref in zip(g["cdf_fit"], g["cdf_u"], g["cdf_nn"], g["cdf_v"]):
        coef = np.zeros(8)
        coef[:4] = fit[:4]
        box = np.array([fit[4], fit[5], 0.0, 1.0])
        assert O.lib().or_cdf_sample(O._p(coef), O._p(box), float(nn), 3, float(u)) == vref


def _fmt(vals, fmt):
    return "".join(fmt % x + "\n" for x in vals)


def test_ballistic_run_matches_reference_files(N, O, golden):
    """Oracle in rand_r mode, one thread, vs the reference binary's `dsmc -n 200 -t 1` outputs:
    density, horizon, ttime and v_record files identical byte for byte."""
    meta, runs = golden["meta"], golden["runs"]
    T = runs["T"]
    np.testing.assert_array_equal(T, cold_T(N))
    p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    S = N.SurfaceInputs(T_map=T)
    r = O.run(p, S, meta["n_particles"], rng=O.RNG_RAND_R, rr_seed=67890, fixed=False, f64=True,
              v_record=True)
    den = f"36\n72\n{p.hd}\n" + _fmt(r["density_f64"].ravel(), "%9.6f")
    hor = "36\n72\n" + _fmt(r["horizon_f64"].ravel(), "%9.6f")
    tt = _fmt(r["ttime"][:5].ravel(), "%9.5f")
    vr = f"{r['n_records']}\n" + "".join(
        "%f %f %f\n%d\n%d\n%d\n" % (*r["v_record"][i], r["v_td"][i], r["v_fd"][i], r["v_ht"][i])
        for i in range(r["n_records"]))
    sha = meta["sha256"]
    for name, text in (("bal_den", den), ("bal_horizon", hor), ("bal_ttime", tt),
                       ("bal_v_record", vr)):
        assert hashlib.sha256(text.encode()).hexdigest() == sha[name], name


def _reference_advanced_inputs(N, O, golden):
    meta, runs = golden["meta"], golden["runs"]
    p = N.params_reference(N.RUNNER_ADVANCED, 36, 72)
    hd, ncell = p.hd, p.ncell
    rec = runs["bal_v_record"]
    cnt = np.zeros(ncell, np.int32)
    sp = np.zeros((ncell, 50))
    for vx, vy, vz, td, fd, ht in rec:
        td, fd, ht = int(td), int(fd), int(ht)
        if not (0 <= td < 36 and 0 <= fd < 72 and 0 <= ht < hd):
            continue
        k = td * 72 * hd + fd * hd + ht
        if cnt[k] < 50:
            sp[k, cnt[k]] = np.sqrt(vx * vx + vy * vy + vz * vz)
            cnt[k] += 1
    coef, box = np.zeros((ncell, 8)), np.zeros((ncell, 4))
    tot, valid = np.zeros(ncell), np.zeros(ncell, np.int32)
    for k in np.nonzero(cnt > 8)[0]:
        c8, b4, t1 = np.zeros(8), np.zeros(4), np.zeros(1)
        valid[k] = O.lib().or_fit_cell_from_samples(O._p(np.ascontiguousarray(sp[k])), int(cnt[k]),
                                                    3, O._p(c8), O._p(b4), O._p(t1))
        coef[k], box[k], tot[k] = c8, b4, t1[0]
    # the phase-1 density as the reference reads it back from its %9.6f file
    nbg = np.array([float("%9.6f" % (x * meta["collision_scale"])) for x in runs["bal_den"]])
    return p, N.CollisionInputs(nbg, coef, box, tot, valid, 3), (sp, cnt)


def test_advanced_run_matches_reference_files(N, O, golden):
    """Oracle vs the reference's `dsmc-adv -n 200 -t 1` with a scaled phase-1 background, so
    that collisions fire (1349 of them): outputs identical byte for byte."""
    meta, runs = golden["meta"], golden["runs"]
    p, col, _ = _reference_advanced_inputs(N, O, golden)
    S = N.SurfaceInputs(T_map=runs["T"])
    r = O.run(p, S, meta["n_particles"], collision=col, rng=O.RNG_RAND_R, rr_seed=98765,
              fixed=False, f64=True)
    assert r["n_collisions"] == meta["adv_collisions"] > 1000
    den = f"36\n72\n{p.hd}\n" + _fmt(r["density_f64"].ravel(), "%9.6f")
    hor = "36\n72\n" + _fmt(r["horizon_f64"].ravel(), "%9.6f")
    tt = _fmt(r["ttime"].ravel(), "%9.5f")
    sha = meta["sha256"]
    for name, text in (("adv_den", den), ("adv_horizon", hor), ("adv_ttime", tt)):
        assert hashlib.sha256(text.encode()).hexdigest() == sha[name], name


def test_fixed_point_and_parallel_oracle_agree(N, O):
    """Philox mode: the fixed-point grids do not depend on the thread count (integer sums)."""
    p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    S = N.SurfaceInputs(T_map=cold_T(N))
    a = O.run(p, S, 300, nthreads=1)
    b = O.run(p, S, 300, nthreads=4)
    np.testing.assert_array_equal(a["density"], b["density"])
    np.testing.assert_array_equal(a["horizon"], b["horizon"])
    np.testing.assert_array_equal(a["ttime"], b["ttime"])


REF_CLI = ROOT / "oracle" / "_ref" / "dsmc_suite"


@pytest.mark.skipif(not REF_CLI.exists(), reason="reference not compiled here")
@pytest.mark.parametrize("n", [1, 57])
def test_live_reference_ballistic_small(N, O, tmp_path, n):
    """Where the reference binary is present, pin further sizes against it directly."""
    T = cold_T(N)
    (tmp_path / "T.dat").write_text("36\n72\n" + "".join(f"{x:.17g}\n" for x in T.ravel()))
    subprocess.run([str(REF_CLI), "dsmc", "-n", str(n), "-t", "1", "-T", str(tmp_path / "T.dat"),
                    "-o", str(tmp_path / "r")], check=True, capture_output=True)
    p = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    r = O.run(p, N.SurfaceInputs(T_map=T), n, rng=O.RNG_RAND_R, rr_seed=67890, fixed=False,
              f64=True)
    den = f"36\n72\n{p.hd}\n" + _fmt(r["density_f64"].ravel(), "%9.6f")
    assert den == (tmp_path / "r_den.dat").read_text()
    assert _fmt(r["ttime"][:5].ravel(), "%9.5f") == (tmp_path / "r_ttime.dat").read_text()


def _thermal_cases(N):
    import sys
    sys.path.insert(0, str(GOLDEN))
    import make_thermal_golden as G
    return G.cases(N)


def test_thermal_oracle_matches_reference(N, O):
    """The oracle's thermal column model equals the reference's thermal_solve bit for bit: against
    the committed fixture (made by the reference build), and live where oracle/_ref exists."""
    g = np.load(GOLDEN / "reference_thermal.npz")
    for name, ftd, ffd, tp, flux in _thermal_cases(N):
        T, h = O.thermal(ftd, ffd, tp, flux)
        np.testing.assert_array_equal(T, g[name])
        assert h >= 3
        live = O.reference_thermal(ftd, ffd, tp, flux)
        if live is not None:
            np.testing.assert_array_equal(T, live)


def test_oracle_problem_setup_is_the_products_bit_for_bit(N):
    """oracle/problems.py builds the CPU arm's inputs without the product library; they must be
    the product's own parameter presets, icosphere and temperature fields, byte for byte."""
    from oracle import problems as OP
    for runner in (N.RUNNER_BALLISTIC, N.RUNNER_ADVANCED):
        for ftd, ffd in ((36, 72), (18, 24)):
            assert bytes(OP.params_reference(runner, ftd, ffd)) == \
                bytes(N.params_reference(runner, ftd, ffd))
        for R, GM, hd, seed in ((470e3, 6.26e10, 50, 20261203), (1561e3, 3.20e12, 20, 7),
                                (1737e3, 4.90e12, 60, 2**63 + 5)):
            assert bytes(OP.params_config(runner, R, GM, hd, seed)) == \
                bytes(N.params_config(runner, R, GM, hd, seed))
    for nlevel in (0, 1, 3):
        a, b = OP.Icosphere(nlevel), N.Icosphere(nlevel)
        for name in ("face_verts", "base_centroid", "split_planes"):
            assert getattr(a, name).tobytes() == getattr(b, name).tobytes(), (nlevel, name)
        for sun, T_ss in (((1.0, 0.0, 0.0), 235.0), ((0.6, 0.8, 0.0), 333.0)):
            assert a.face_temperature(sun, T_ss, 110.0).tobytes() == \
                b.face_temperature(sun, T_ss, 110.0).tobytes()
    for sun in ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0)):
        assert OP.latlon_temperature(36, 72, sun, 235.0, 60.0).tobytes() == \
            N.latlon_temperature(36, 72, sun, 235.0, 60.0).tobytes()


def test_reference_arm_loads_only_oracle_libraries(tmp_path):
    """The timed CPU arm of bench.py builds its workload with oracle/problems.py and runs the
    oracle port: the product library must not be mapped into that process."""
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import bench\n"
            "r = bench.cpu_oracle_rate(0.2, 2, 300)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libdsmc_b200' not in maps, 'product library loaded'\n"
            "assert 'liboracle.so' in maps\n"
            "assert 'dsmc_suite_b200' not in sys.modules\n"
            "print(r[2])\n" % str(ROOT))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    assert int(out.stdout.split()[-1]) > 0


def test_oracle_energy_drift_guard(O):
    """The per-hop energy-drift guard of the oracle: the config workloads' hops at dt = 2 s stay
    inside drift_tol * GM / R (the reference's integrator drifts by ~1e-3 GM / R over a hop), a
    ten times larger step flags many hops, and drift_tol = 0 turns the count off."""
    import math
    from oracle import problems as OP
    ico = OP.Icosphere(3)
    S = OP.SurfaceInputs(ico=ico, face_T=ico.face_temperature())
    for R, GM in ((470e3, 6.26e10), (1737e3, 4.90e12)):
        p = OP.params_config(OP.RUNNER_BALLISTIC, R, GM, 50, 11)
        assert O.run(p, S, 1500, nthreads=4, particles=False)["n_drift_flagged"] == 0
        p.dt_step = 20.0
        p.wdecay = math.exp(-p.dt_step / p.lifetime)
        big = O.run(p, S, 1500, nthreads=4, particles=False)
        assert big["n_drift_flagged"] > 500
        p.drift_tol = 0.0
        assert O.run(p, S, 300, nthreads=4, particles=False)["n_drift_flagged"] == 0
