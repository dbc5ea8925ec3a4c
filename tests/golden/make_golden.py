"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs in the build container, where the reference sources exist and oracle/Makefile has compiled
them into oracle/_ref/ (the unmodified reference CLI `dsmc_suite`, its `test_verlet`, and
`libdsmcref.so` with its scalar functions). Nothing here is needed at test time: the tests read
the .npz / .json files this script writes.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import re
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = ROOT / "oracle" / "_ref"
sys.path.insert(0, str(ROOT))

FTD, FFD = 36, 72
N_PARTICLES = 200
COLLISION_SCALE = 1e12   # phase-1 density scale that makes the collision branch fire


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


def synthetic_T() -> np.ndarray:
    """36 x 72 map T = max(60, 235 cos(z)^(1/4)) with fully cold polar rows, so that the
    reference's freeze scan and its permanent freeze both fire."""
    from dsmc_suite_b200 import _native as N
    T = N.latlon_temperature(FTD, FFD, T_ss=235.0, T_floor=60.0)
    T[:2, :] = 50.0
    T[-2:, :] = 50.0
    return T


def write_T(path: Path, T: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write(f"{T.shape[0]}\n{T.shape[1]}\n")
        f.writelines(f"{x:.17g}\n" for x in T.ravel())


def sha(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


def load_vals(path: Path, skip: int) -> np.ndarray:
    return np.array(path.read_text().split()[skip:], dtype=np.float64)


def run_reference_cli(tmp: Path, T: np.ndarray) -> dict:
    write_T(tmp / "T.dat", T)
    cli = str(REF / "dsmc_suite")
    subprocess.run([cli, "dsmc", "-n", str(N_PARTICLES), "-t", "1", "-T", str(tmp / "T.dat"),
                    "-o", str(tmp / "p1")], check=True, capture_output=True)
    den1 = load_vals(tmp / "p1_den.dat", 3)
    with open(tmp / "p1s_den.dat", "w") as f:
        f.write(f"{FTD}\n{FFD}\n100\n")
        f.writelines("%9.6f\n" % (x * COLLISION_SCALE) for x in den1)
    out = subprocess.run([cli, "dsmc-adv", "-n", str(N_PARTICLES), "-t", "1", "-T",
                          str(tmp / "T.dat"), "-d", str(tmp / "p1s_den.dat"), "-v",
                          str(tmp / "p1_v_record.dat"), "-o", str(tmp / "p2")],
                         check=True, capture_output=True, text=True).stdout
    m = re.search(r"Total collisions: (\d+)", out)
    vr = (tmp / "p1_v_record.dat").read_text().split()
    nrec = int(vr[0])
    rec = np.array(vr[1:], dtype=np.float64).reshape(nrec, 6)
    return {
        "T": T,
        "bal_den": den1, "bal_horizon": load_vals(tmp / "p1_horizon.dat", 2),
        "bal_ttime": load_vals(tmp / "p1_ttime.dat", 0), "bal_v_record": rec,
        "adv_den": load_vals(tmp / "p2_den.dat", 3),
        "adv_horizon": load_vals(tmp / "p2_horizon.dat", 2),
        "adv_ttime": load_vals(tmp / "p2_ttime.dat", 0),
        "adv_collisions": int(m.group(1)),
        "sha": {k: sha(tmp / f) for k, f in [("bal_den", "p1_den.dat"),
                                              ("bal_horizon", "p1_horizon.dat"),
                                              ("bal_ttime", "p1_ttime.dat"),
                                              ("bal_v_record", "p1_v_record.dat"),
                                              ("adv_den", "p2_den.dat"),
                                              ("adv_horizon", "p2_horizon.dat"),
                                              ("adv_ttime", "p2_ttime.dat")]},
    }


def scalar_vectors() -> dict:
    L = C.CDLL(str(REF / "libdsmcref.so"))
    L.verlet_step.restype = C.c_int
    L.verlet_step.argtypes = [C.POINTER(Particle), C.POINTER(PhysicsParams), C.c_double,
                              C.POINTER(Vec3), C.POINTER(C.c_double)]
    L.grid_spherical_to_index.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int,
                                          C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.grid_exp_ht_index.restype = C.c_int
    L.grid_exp_ht_index.argtypes = [C.c_double] * 4
    L.velocity_table_init.argtypes = [C.POINTER(VelocityTable), C.c_double, C.c_double, C.c_double]
    L.velocity_sample.restype = C.c_double
    L.velocity_sample.argtypes = [C.POINTER(VelocityTable), C.c_double, C.POINTER(C.c_uint)]
    L.collision_sample_speed.restype = C.c_double
    L.collision_sample_speed.argtypes = [C.POINTER(PolyFit), C.c_double, C.c_int]
    L.polyfit.restype = C.c_int
    L.polyfit.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_int,
                          C.POINTER(C.c_double)]
    rng = np.random.default_rng(20261203)
    out: dict = {}

    # verlet_step: 64 fed states x 400 steps with the reference ballistic parameters
    pp = PhysicsParams(G=6.67e-11, M=9.39e20, Radii=476.2e3, max_height=476.2e3 * 11.0)
    GM = pp.G * pp.M
    n, steps, h = 64, 400, 5.0
    r0 = pp.Radii * rng.uniform(1.0005, 1.2, n)
    th = np.arcsin(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    s0 = np.stack([r0 * np.cos(th) * np.sin(ph), r0 * np.cos(th) * np.cos(ph), r0 * np.sin(th)], 1)
    v0 = rng.normal(0, 150.0, (n, 3)) + s0 / np.linalg.norm(s0, axis=1)[:, None] * 200.0
    fin_s, fin_v, fin_oa, stat, taken, ds_last = [], [], [], [], [], []
    for i in range(n):
        p = Particle()
        p.pos = Vec3(*s0[i])
        p.vel = Vec3(*v0[i])
        R = np.sqrt(s0[i][0] * s0[i][0] + s0[i][1] * s0[i][1] + s0[i][2] * s0[i][2])
        oa = Vec3(*(GM * s0[i][k] / (R * R * R) for k in range(3)))
        ds = C.c_double()
        st, k = 0, 0
        while k < steps and st == 0:
            st = L.verlet_step(C.byref(p), C.byref(pp), h, C.byref(oa), C.byref(ds))
            k += 1
        fin_s.append([p.pos.x, p.pos.y, p.pos.z])
        fin_v.append([p.vel.x, p.vel.y, p.vel.z])
        fin_oa.append([oa.x, oa.y, oa.z])
        stat.append(st)
        taken.append(k)
        ds_last.append(ds.value)
    out.update(verlet_s0=s0, verlet_v0=v0, verlet_h=h, verlet_steps=steps, verlet_GM=GM,
               verlet_Radii=pp.Radii, verlet_max_height=pp.max_height,
               verlet_s=np.array(fin_s), verlet_v=np.array(fin_v), verlet_oa=np.array(fin_oa),
               verlet_status=np.array(stat), verlet_taken=np.array(taken),
               verlet_ds=np.array(ds_last))

    # grid_spherical_to_index, including exact cell boundaries
    thi = np.concatenate([rng.uniform(-np.pi / 2, np.pi / 2, 2000),
                          np.arange(FTD + 1) / FTD * np.pi - np.pi / 2])
    fi = np.concatenate([rng.uniform(0, 2 * np.pi, 2000), np.arange(FTD + 1) / FFD * 2 * np.pi])
    td, fd = C.c_int(), C.c_int()
    idx = []
    for a, b in zip(thi, fi):
        L.grid_spherical_to_index(a, b, FTD, FFD, C.byref(td), C.byref(fd))
        idx.append((td.value, fd.value))
    out.update(index_thi=thi, index_fi=fi, index_td_fd=np.array(idx))

    # grid_exp_ht_index with the advanced runner's grid (advanced.c:148-152)
    R, hmax, a2, hd = 476.2e3, 3e6 * np.sqrt(2.0), 0.04, 50
    unih = (hmax - R) / (pow(1.0 + a2, hd) - 1.0) * a2
    radii = np.concatenate([R + rng.uniform(0, hmax - R, 2000),
                            [R + (pow(1 + a2, k) - 1) / a2 * unih for k in range(hd + 1)]])
    out.update(expht_radii=radii, expht_unih=unih,
               expht_index=np.array([L.grid_exp_ht_index(r, R, unih, a2) for r in radii]))

    # velocity table and velocity_sample sequences (seed 42, as tests/test_verlet.c:75)
    vt = VelocityTable()
    L.velocity_table_init(C.byref(vt), 18e-3, 6.02e23, 1.38e-23)
    samples = {}
    for T in (20.0, 95.0, 100.0, 150.0, 200.0, 219.9, 220.0, 260.0):
        seed = C.c_uint(42)
        samples[T] = [L.velocity_sample(C.byref(vt), T, C.byref(seed)) for _ in range(200)]
    out.update(vt_speeds=np.array(vt.speeds), vt_count=np.array(vt.count),
               vt_temps=np.array(vt.temps), vs_T=np.array(list(samples)),
               vs_values=np.array(list(samples.values())))

    # polyfit on noisy cubic-like data, degrees 1..6
    pf_x, pf_y, pf_c = [], [], []
    for deg in range(1, 7):
        x = np.sort(rng.uniform(100, 600, 25))
        y = 50 - 0.1 * x + rng.normal(0, 1, 25)
        c = (C.c_double * 7)()
        L.polyfit(x.ctypes.data_as(C.POINTER(C.c_double)),
                  y.ctypes.data_as(C.POINTER(C.c_double)), 25, deg, c)
        pf_x.append(x)
        pf_y.append(y)
        pf_c.append(list(c))
    out.update(polyfit_x=np.array(pf_x), polyfit_y=np.array(pf_y), polyfit_c=np.array(pf_c))

    # collision_sample_speed on fitted reverse-cumulative speed distributions
    cs_fit, cs_u, cs_nn, cs_v = [], [], [], []
    for _ in range(40):
        nn = int(rng.integers(9, 51))
        sp = np.sort(rng.uniform(100, 700, nn))
        nb = max(4, (nn + 1) // 2)
        dv = (sp[-1] - sp[0]) / nb
        xx = sp[0] + (np.arange(nb) + 0.5) * dv
        yy = np.zeros(nb)
        for v in sp:
            yy[min(nb - 1, max(0, int((v - sp[0]) / dv)))] += 1
        yy2 = np.cumsum(yy[::-1])[::-1].copy()
        c = (C.c_double * 7)()
        L.polyfit(xx.ctypes.data_as(C.POINTER(C.c_double)),
                  yy2.ctypes.data_as(C.POINTER(C.c_double)), nb, 3, c)
        pf = PolyFit()
        for k in range(4):
            pf.coeffs[k] = c[k]
        pf.min_v, pf.max_v, pf.valid = sp[0], sp[-1], 1
        u = float(rng.uniform())
        cs_fit.append([c[0], c[1], c[2], c[3], sp[0], sp[-1]])
        cs_u.append(u)
        cs_nn.append(nn)
        cs_v.append(L.collision_sample_speed(C.byref(pf), u, nn))
    out.update(cdf_fit=np.array(cs_fit), cdf_u=np.array(cs_u), cdf_nn=np.array(cs_nn),
               cdf_v=np.array(cs_v))
    return out


def test_verlet_kats() -> dict:
    txt = subprocess.run([str(REF / "test_verlet")], capture_output=True, text=True).stdout
    E = re.search(r"E0 = ([-\d.e+]+), E1 = ([-\d.e+]+), rel_error = ([-\d.e+]+)", txt)
    mv = re.search(r"Mean velocity at 200K: ([\d.]+)", txt)
    co = re.search(r"Coefficients: ([-\d. ]+)\n", txt)
    pv = re.search(r"polyval\(5\) = ([-\d.]+)", txt)
    return {"E0": float(E.group(1)), "E1": float(E.group(2)), "rel_error": float(E.group(3)),
            "mean_v_200K": float(mv.group(1)),
            "coefficients": [float(x) for x in co.group(1).split()],
            "polyval5": float(pv.group(1)), "stdout": txt}


def main() -> None:
    if not (REF / "dsmc_suite").exists():
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` first")
    with tempfile.TemporaryDirectory() as d:
        res = run_reference_cli(Path(d), synthetic_T())
    sha_map = res.pop("sha")
    ncol = res.pop("adv_collisions")
    np.savez_compressed(HERE / "reference_runs.npz", **res)
    np.savez_compressed(HERE / "reference_scalars.npz", **scalar_vectors())
    meta = {"n_particles": N_PARTICLES, "ftd": FTD, "ffd": FFD,
            "collision_scale": COLLISION_SCALE, "adv_collisions": ncol, "sha256": sha_map,
            "rand_r_seeds": {"ballistic": 67890, "advanced": 98765},
            "test_verlet": test_verlet_kats()}
    (HERE / "reference_meta.json").write_text(json.dumps(meta, indent=1, sort_keys=True))
    print("wrote", sorted(p.name for p in HERE.glob("reference_*")))


if __name__ == "__main__":
    main()
