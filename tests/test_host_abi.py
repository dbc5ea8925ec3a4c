"""Host side of the product library, no GPU needed: the C ABI exports, the reference-model
presets, the reference's kept scalar entry points (bit for bit against the reference's own
functions), the icosphere surface, the .dat formats and the CLI's error paths."""
from __future__ import annotations

import ctypes as C
import math
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cold_T

INCLUDE = ROOT / "include"


def declared_functions():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"static inline[^{]*\{[^}]*\}", "", text)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(N):
    lib = N.lib()
    names = declared_functions()
    assert {"dsmc_ctx_create", "verlet_step", "run_ballistic", "write_density_dat"} <= names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows every dsmc_* function the C header declares
    bound = {s[0] for s in N.SIGNATURES}
    assert {n for n in names if n.startswith("dsmc_")} <= bound


def test_reference_presets(N):
    b = N.params_reference(N.RUNNER_BALLISTIC, 36, 72)
    G, M, R = 6.67e-11, 9.39e20, 476.2e3
    assert b.GM == G * M and b.Radii == R and b.ve == math.sqrt(2.0 * G * M / R)
    assert b.dt_step == 5.0 and b.hd == 100 and not b.use_exp_grid
    assert b.unih == R * 0.1 and b.max_height == R * 0.1 * 100 + R
    assert b.wdecay == math.exp(-5.0 / (1.0 / 1.02e-5 * (2.8 * 2.8)))
    assert b.dt_rot == 9.07417 * 3600.0 / 72 and b.skip_first_deposit == 1
    a = N.params_reference(N.RUNNER_ADVANCED, 36, 72)
    hmax = 3e6 * math.sqrt(2.0)
    assert a.dt_step == 0.5 and a.hd == 50 and a.use_exp_grid and a.alpha2 == 0.04
    assert a.unih == (hmax - R) / (pow(1.04, 50) - 1.0) * 0.04
    assert a.cross_section == 1e-19 and a.collide_ht_max == 50 // 3
    c = N.params_config(N.RUNNER_BALLISTIC)
    assert c.Radii == 470e3 and c.GM == 6.26e10 and c.dt_step == 2.0
    assert c.life_step_cap == 20000 and c.lifetime == 2.6e5 and c.hd == 50
    assert abs(c.max_height - 4.7e6) < 1e-6 and abs(c.cross_section - math.pi * 4.6e-10 ** 2) < 1e-30


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class Particle(C.Structure):
    _fields_ = [("pos", Vec3), ("vel", Vec3), ("weight", C.c_double), ("td", C.c_int),
                ("fd", C.c_int), ("ht", C.c_int), ("flight_time", C.c_double),
                ("collision_count", C.c_int)]


class PhysicsParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("G", "M", "k_B", "mmass", "mole", "Radii", "ve",
                                          "lifetime", "P", "cross_section", "alpha", "dt_step",
                                          "dt_rot", "max_height", "unih", "alpha2")] + \
               [("use_exp_grid", C.c_int)]


class VelocityTable(C.Structure):
    _fields_ = [("temps", C.c_double * 23), ("speeds", (C.c_double * 1000) * 23),
                ("count", C.c_int * 23)]


class PolyFit(C.Structure):
    _fields_ = [("coeffs", C.c_double * 4), ("min_v", C.c_double), ("max_v", C.c_double),
                ("valid", C.c_int)]


def test_kept_verlet_step_bit_exact(N, golden):
    L = N.lib()
    L.verlet_step.restype = C.c_int
    L.verlet_step.argtypes = [C.POINTER(Particle), C.POINTER(PhysicsParams), C.c_double,
                              C.POINTER(Vec3), C.POINTER(C.c_double)]
    g = golden["scalars"]
    pp = PhysicsParams(G=6.67e-11, M=9.39e20, Radii=float(g["verlet_Radii"]),
                       max_height=float(g["verlet_max_height"]))
    for i in range(len(g["verlet_s0"])):
        p = Particle()
        p.pos = Vec3(*g["verlet_s0"][i])
        p.vel = Vec3(*g["verlet_v0"][i])
        s = g["verlet_s0"][i]
        R = math.sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2])
        oa = Vec3(*(pp.G * pp.M * s[k] / (R * R * R) for k in range(3)))
        ds = C.c_double()
        st, k = 0, 0
        while k < g["verlet_steps"] and st == 0:
            st = L.verlet_step(C.byref(p), C.byref(pp), float(g["verlet_h"]), C.byref(oa),
                               C.byref(ds))
            k += 1
        assert (st, k) == (g["verlet_status"][i], g["verlet_taken"][i])
        assert [p.pos.x, p.pos.y, p.pos.z] == list(g["verlet_s"][i])
        assert [p.vel.x, p.vel.y, p.vel.z] == list(g["verlet_v"][i])
        assert [oa.x, oa.y, oa.z] == list(g["verlet_oa"][i])
        assert ds.value == g["verlet_ds"][i]


def test_kept_velocity_and_grid_functions(N, golden):
    L = N.lib()
    g = golden["scalars"]
    vt = VelocityTable()
    L.velocity_table_init.argtypes = [C.POINTER(VelocityTable), C.c_double, C.c_double, C.c_double]
    L.velocity_table_init(C.byref(vt), 18e-3, 6.02e23, 1.38e-23)
    np.testing.assert_array_equal(np.array(vt.speeds), g["vt_speeds"])
    np.testing.assert_array_equal(np.array(vt.count), g["vt_count"])
    L.velocity_sample.restype = C.c_double
    L.velocity_sample.argtypes = [C.POINTER(VelocityTable), C.c_double, C.POINTER(C.c_uint)]
    for T, ref in zip(g["vs_T"], g["vs_values"]):
        seed = C.c_uint(42)
        assert [L.velocity_sample(C.byref(vt), float(T), C.byref(seed)) for _ in ref] == list(ref)
    L.grid_spherical_to_index.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int,
                                          C.POINTER(C.c_int), C.POINTER(C.c_int)]
    td, fd = C.c_int(), C.c_int()
    for a, b, ref in zip(g["index_thi"], g["index_fi"], g["index_td_fd"]):
        L.grid_spherical_to_index(float(a), float(b), 36, 72, C.byref(td), C.byref(fd))
        assert (td.value, fd.value) == tuple(ref)
    L.grid_exp_ht_index.restype = C.c_int
    L.grid_exp_ht_index.argtypes = [C.c_double] * 4
    for r, ref in zip(g["expht_radii"], g["expht_index"]):
        assert L.grid_exp_ht_index(float(r), 476.2e3, float(g["expht_unih"]), 0.04) == ref


def test_kept_polyfit_and_collision_functions(N, golden):
    L = N.lib()
    g = golden["scalars"]
    L.polyfit.restype = C.c_int
    L.polyfit.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_int,
                          C.POINTER(C.c_double)]
    for deg, (x, y, cref) in enumerate(zip(g["polyfit_x"], g["polyfit_y"], g["polyfit_c"]), 1):
        c = (C.c_double * 7)()
        x, y = np.ascontiguousarray(x), np.ascontiguousarray(y)
        assert L.polyfit(N.ptr(x), N.ptr(y), len(x), deg, c) == 0
        assert list(c)[:deg + 1] == list(cref[:deg + 1])
    L.collision_sample_speed.restype = C.c_double
    L.collision_sample_speed.argtypes = [C.POINTER(PolyFit), C.c_double, C.c_int]
    for fit, u, nn, vref in zip(g["cdf_fit"], g["cdf_u"], g["cdf_nn"], g["cdf_v"]):
        pf = PolyFit()
        for k in range(4):
            pf.coeffs[k] = fit[k]
        pf.min_v, pf.max_v, pf.valid = fit[4], fit[5], 1
        assert L.collision_sample_speed(C.byref(pf), float(u), int(nn)) == vref
    L.collision_execute.argtypes = [C.POINTER(Vec3), Vec3]
    v = Vec3(1.0, 2.0, 3.0)
    L.collision_execute(C.byref(v), Vec3(4.0, -2.0, 0.5))
    assert (v.x, v.y, v.z) == (1.5 * 1 + 0.5 * 4, 1.5 * 2 - 0.5 * 2, 1.5 * 3 + 0.5 * 0.5)


def test_icosphere_surface(N, O):
    ico = N.Icosphere(3)
    assert ico.nface == 1280 and ico.nnode == 420
    v = ico.face_verts.reshape(-1, 3)
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
    assert len(np.unique(np.round(v, 12), axis=0)) == 642
    a, b, c = v[0::3], v[1::3], v[2::3]
    n = np.cross(b - a, c - a)
    assert (np.einsum("ij,ij->i", n, a + b + c) > 0).all()     # all faces outward
    area = 0.5 * np.linalg.norm(n, axis=1).sum()
    assert 0.98 * 4 * np.pi < area < 4 * np.pi
    # the tree descent agrees with the oracle's brute-force cone test
    S = N.SurfaceInputs(ico=ico, face_T=np.zeros(1280))
    rng = np.random.default_rng(5)
    L = O.lib()
    for _ in range(3000):
        p = rng.normal(size=3)
        p /= np.linalg.norm(p)
        assert ico.locate(p) == L.or_locate_face(C.addressof(S.struct), O._p(np.ascontiguousarray(p)))
    T = ico.face_temperature(T_ss=235.0, T_floor=110.0)
    assert T.min() == 110.0 and 230 < T.max() <= 235.0
    cdf, rate = ico.source_cdf(T)
    assert cdf[-1] == 1.0 and np.all(np.diff(cdf) >= 0) and rate > 0
    # sublimation flux rises steeply with temperature (Antoine vapour pressure)
    f = N.lib().dsmc_sublimation_flux
    assert f(110.0, 2.99e-26) < 1e-6 * f(235.0, 2.99e-26)


def test_latlon_temperature_convention(N):
    T = N.latlon_temperature(36, 72, T_ss=235.0, T_floor=110.0)
    # sub-solar point on +x: longitude pi/2 (column 17/18 edge), equator
    assert T[17:19, 17:19].min() > 230 and T[:, 45:63].max() == 110.0


def test_dat_formats_round_trip_and_bytes(N, tmp_path, golden):
    L = N.lib()
    L.write_density_dat.argtypes = [C.c_char_p, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int]
    L.read_density_dat.restype = C.POINTER(C.c_double)
    L.read_density_dat.argtypes = [C.c_char_p] + [C.POINTER(C.c_int)] * 3 + [C.c_int]
    runs = golden["runs"]
    den = np.ascontiguousarray(runs["bal_den"])
    path = str(tmp_path / "d.dat").encode()
    assert L.write_density_dat(path, N.ptr(den), 36, 72, 100) == 0
    import hashlib
    assert hashlib.sha256((tmp_path / "d.dat").read_bytes()).hexdigest() == \
        golden["meta"]["sha256"]["bal_den"]
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    q = L.read_density_dat(path, C.byref(a), C.byref(b), C.byref(c), 1)
    assert (a.value, b.value, c.value) == (36, 72, 100)
    np.testing.assert_array_equal(np.ctypeslib.as_array(q, shape=(den.size,)), den)
    # a short file is rejected instead of being half read
    (tmp_path / "short.dat").write_text("36\n72\n100\n1.0\n2.0\n")
    assert not L.read_density_dat(str(tmp_path / "short.dat").encode(), C.byref(a), C.byref(b),
                                  C.byref(c), 1)
    L.read_temperature_dat.restype = C.POINTER(C.c_double)
    L.read_temperature_dat.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    assert not L.read_temperature_dat(str(tmp_path / "missing.dat").encode(), C.byref(a), C.byref(b))


def test_grids_side_car_round_trip(N, tmp_path):
    """write_grids_bin + read_grids_bin give back the exact grids and FP64 rows; the values
    count / fixed_scale print to the same text as write_density_dat / write_ttime_dat; a
    truncated or foreign file is rejected."""
    from dsmc_suite_b200.sidecar import read_grids_bin
    L = N.lib()
    u64 = C.POINTER(C.c_uint64)
    L.write_grids_bin.argtypes = [C.c_char_p, u64, u64, C.POINTER(C.c_double)] + [C.c_int] * 5 + \
        [C.c_double]
    rng = np.random.default_rng(7)
    ftd, ffd, hd, nrows, n = 3, 5, 4, 5, 11
    den = rng.integers(0, 1 << 40, hd * ftd * ffd, dtype=np.uint64)
    hor = rng.integers(0, 1 << 30, ftd * ffd, dtype=np.uint64)
    tt = rng.normal(size=(nrows, n)) * 1e4
    path = tmp_path / "r_grids.bin"
    assert L.write_grids_bin(str(path).encode(), den.ctypes.data_as(u64), hor.ctypes.data_as(u64),
                             N.ptr(tt), ftd, ffd, hd, nrows, n, N.FIXED_SCALE) == 0
    g = read_grids_bin(path)
    assert (g["ftd"], g["ffd"], g["hd"], g["nrows"], g["totaln"]) == (ftd, ffd, hd, nrows, n)
    np.testing.assert_array_equal(g["density"], den)
    np.testing.assert_array_equal(g["horizon"], hor)
    np.testing.assert_array_equal(g["ttime"], tt)
    L.write_density_dat.argtypes = [C.c_char_p, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int]
    dd = np.ascontiguousarray(den / g["fixed_scale"])
    assert L.write_density_dat(str(tmp_path / "r_den.dat").encode(), N.ptr(dd), ftd, ffd, hd) == 0
    text = (tmp_path / "r_den.dat").read_text().split("\n")[3:-1]
    assert text == ["%9.6f" % x for x in g["density"] / g["fixed_scale"]]
    L.write_grids_bin(str(path).encode(), den.ctypes.data_as(u64), hor.ctypes.data_as(u64), None,
                      ftd, ffd, hd, nrows, 0, N.FIXED_SCALE)
    assert read_grids_bin(path)["ttime"].shape == (nrows, 0)
    (tmp_path / "cut.bin").write_bytes(path.read_bytes()[:-8])
    with pytest.raises(ValueError):
        read_grids_bin(tmp_path / "cut.bin")
    (tmp_path / "bad.bin").write_bytes(b"XXXXXXXX" + path.read_bytes()[8:])
    with pytest.raises(ValueError):
        read_grids_bin(tmp_path / "bad.bin")


def test_cli_usage_and_out_of_scope_commands(built):
    cli = ROOT / "dsmc_suite_b200" / "bin" / "dsmc_suite"
    r = subprocess.run([str(cli)], capture_output=True, text=True)
    assert r.returncode == 1 and "dsmc-adv" in r.stdout
    r = subprocess.run([str(cli), "raytrace"], capture_output=True, text=True)
    assert r.returncode == 1 and "requires -m" in r.stderr
    r = subprocess.run([str(cli), "bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown command" in r.stderr


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_fails_loudly(N):
    from dsmc_suite_b200 import Context, DsmcError
    with pytest.raises(DsmcError) as e:
        Context(0)
    assert e.value.status == -3   # DSMC_ERR_NO_DEVICE: there is no CPU fallback


def test_cold_map_has_permanent_freeze_rows(N):
    T = cold_T(N)
    assert (T[:2] < 100).all() and (T[2:-2] >= 100).any(axis=1).all()


def test_number_density_fp64_behind_the_c_abi(N):
    """dsmc_number_density_host turns a fixed-point grid into molecules per m^3 in FP64; it must
    agree with the host formula of workloads.number_density (physical volumes) and, with the
    reference's volume convention, use the kept grid_compute_volume_* cells."""
    from dsmc_suite_b200 import workloads as W
    rng = np.random.default_rng(5)
    for p in (N.params_config(N.RUNNER_BALLISTIC), N.params_config(N.RUNNER_ADVANCED, 1561e3, 3.2e12, 20),
              N.params_reference(N.RUNNER_BALLISTIC, 36, 72), N.params_reference(N.RUNNER_ADVANCED, 36, 72)):
        fx = rng.integers(0, 2**40, size=(p.hd, p.ftd, p.ffd), dtype=np.uint64)
        fx[0, 0, :3] = 0
        n, rate = 123457, 2.0e26
        got = N.number_density(p, fx, n, rate)
        want = W.number_density(p, fx, n, rate)
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=0)
        assert (got[0, 0, :3] == 0).all()
        # volumes: physical cells add up to the shell volume between R and max_height
        vol = N.cell_volumes(p)
        r_top = W.shell_radii(p)[-1]
        assert abs(vol.sum() / (4.0 / 3.0 * np.pi * (r_top**3 - p.Radii**3)) - 1.0) < 1e-12
        # the reference's own convention, through the kept entry points
        vref = N.cell_volumes(p, N.VOLUME_REFERENCE)
        g = N.SphericalGrid(ftd=p.ftd, ffd=p.ffd, hd=p.hd, volume=N.ptr(np.zeros(1)))
        v2 = np.zeros(p.ncell)
        g.volume = N.ptr(v2)
        L = N.lib()
        if p.use_exp_grid:
            L.grid_compute_volume_exp(C.byref(g), C.c_double(p.Radii), C.c_double(p.unih),
                                      C.c_double(p.alpha2))
        else:
            L.grid_compute_volume_uniform(C.byref(g), C.c_double(p.Radii), C.c_double(p.unih))
        assert vref.ravel().tobytes() == v2.tobytes()
        ref_nd = N.number_density(p, fx, n, rate, N.VOLUME_REFERENCE)
        np.testing.assert_allclose(ref_nd * vref, got * vol, rtol=1e-13)
    with pytest.raises(N.DsmcError):
        N.number_density(p, fx, 0, rate)
    with pytest.raises(N.DsmcError):
        N.number_density(p, fx, n, rate, 7)
