"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) - TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker; the
product (dsmc_suite_b200/) never imports it. build() compiles oracle/dsmc_oracle.c with gcc, and
build_ref() compiles the reference's own sources into oracle/_ref/ when the reference tree is
present.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
RNG_RAND_R, RNG_PHILOX = 0, 1


def build(ref_root: str | None = None) -> None:
    """Build liboracle.so; also oracle/_ref when the reference sources exist: ref_root, else
    $DSMC_REFERENCE_ROOT, else a checkout named `reference` beside this repository."""
    env = dict(os.environ)
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True, env=env)
    ref = ref_root or os.environ.get("DSMC_REFERENCE_ROOT") or str(HERE.parent.parent / "reference")
    if Path(ref, "src", "dsmc", "ballistic.c").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={ref}"], check=True, env=env)


class VTable(C.Structure):
    _fields_ = [("temps", C.c_double * 23), ("speeds", (C.c_double * 1000) * 23),
                ("count", C.c_int * 23)]


class Outputs(C.Structure):
    _fields_ = [
        ("density_f64", C.POINTER(C.c_double)), ("density_fx", C.POINTER(C.c_uint64)),
        ("horizon_f64", C.POINTER(C.c_double)), ("horizon_fx", C.POINTER(C.c_uint64)),
        ("ttime", C.POINTER(C.c_double)), ("fate", C.POINTER(C.c_int32)),
        ("steps", C.POINTER(C.c_int64)), ("speed_hist", C.POINTER(C.c_uint64)),
        ("v_record", C.POINTER(C.c_double)), ("v_td", C.POINTER(C.c_int32)),
        ("v_fd", C.POINTER(C.c_int32)), ("v_ht", C.POINTER(C.c_int32)),
        ("v_count_nn", C.POINTER(C.c_int32)), ("v_cap", C.c_int64), ("n_records", C.c_int64),
        ("total_steps", C.c_int64), ("n_escaped", C.c_int64), ("n_collisions", C.c_int64),
        ("n_bound_launch", C.c_int64), ("n_drift_flagged", C.c_int64),
    ]


_lib = None


def lib() -> C.CDLL:
    """liboracle.so with its signatures. Structure arguments (dsmc_params, dsmc_surface,
    dsmc_collision, ThermalParams) are passed by address, so callers may use the product's ctypes
    structures (tests) or the oracle's own (oracle/problems.py, the timed CPU arm, which must not
    load the product library)."""
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        D = C.POINTER(C.c_double)
        V = C.c_void_p
        L.or_run.restype = C.c_int
        L.or_run.argtypes = [V, V, V, C.POINTER(VTable), C.c_int, C.c_uint, C.c_int64, C.c_int64,
                             C.c_int, C.POINTER(Outputs)]
        L.or_philox4x32.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]
        L.or_verlet_step.restype = C.c_int
        L.or_verlet_step.argtypes = [D, D, D, C.c_double, C.c_double, C.c_double, C.c_double, D]
        L.or_spherical_to_index.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int,
                                            C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.or_exp_ht_index.restype = C.c_int
        L.or_exp_ht_index.argtypes = [C.c_double] * 5
        L.or_velocity_table_init.argtypes = [C.POINTER(VTable), C.c_double, C.c_double, C.c_double]
        L.or_velocity_sample_word.restype = C.c_double
        L.or_velocity_sample_word.argtypes = [C.POINTER(VTable), C.c_double, C.c_uint32]
        L.or_cdf_sample.restype = C.c_double
        L.or_cdf_sample.argtypes = [D, D, C.c_double, C.c_int, C.c_double]
        L.or_thermal_solve.restype = C.c_int
        L.or_thermal_solve.argtypes = [C.c_int, C.c_int, V, D, D, C.POINTER(C.c_int)]
        L.or_shadow_flux.restype = C.c_int
        L.or_shadow_flux.argtypes = [C.c_int, D, C.c_int, C.POINTER(C.c_int32), D, C.c_double,
                                     C.c_int, C.c_int, D, C.c_int]
        L.or_polyfit.restype = C.c_int
        L.or_polyfit.argtypes = [D, D, C.c_int, C.c_int, D]
        L.or_fit_cell_from_samples.restype = C.c_int
        L.or_fit_cell_from_samples.argtypes = [D, C.c_int, C.c_int, D, D, D]
        L.or_fit_cell_from_hist.restype = C.c_int
        L.or_fit_cell_from_hist.argtypes = [C.POINTER(C.c_uint64), C.c_int, C.c_double, C.c_int,
                                            D, D, D]
        L.or_locate_face.restype = C.c_int
        L.or_locate_face.argtypes = [V, D]
        _lib = L
    return _lib


def _addr(struct) -> int | None:
    return None if struct is None else C.addressof(struct)


def _p(a, t=C.c_double):
    if a is None:
        return C.POINTER(t)()
    return a.ctypes.data_as(C.POINTER(t))


def vtable(mmass=18e-3, mole=6.02e23, k_B=1.38e-23) -> VTable:
    vt = VTable()
    lib().or_velocity_table_init(C.byref(vt), mmass, mole, k_B)
    return vt


def philox(ctr, key) -> list[int]:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().or_philox4x32(c, k, o)
    return list(o)


def run(params, surface, n: int, collision=None, rng: int = RNG_PHILOX, rr_seed: int = 67890,
        pid_begin: int = 0, nthreads: int = 1, fixed: bool = True, f64: bool = False,
        particles: bool = True, v_record: bool = False, speed_hist: bool = False) -> dict:
    """Run the oracle over particles [pid_begin, pid_begin + n); returns numpy results.

    params is a dsmc_params ctypes structure and surface / collision own a dsmc_surface /
    dsmc_collision in their `.struct` (the product's SurfaceInputs / CollisionInputs, or
    oracle.problems.SurfaceInputs)."""
    p = params
    ncell, nh = p.hd * p.ftd * p.ffd, p.ftd * p.ffd
    o = Outputs()
    res: dict = {}
    keep = []

    def arr(name, shape, dtype, field, ctype):
        a = np.zeros(shape, dtype=dtype)
        res[name] = a
        keep.append(a)
        setattr(o, field, _p(a, ctype))

    if fixed:
        arr("density", (p.hd, p.ftd, p.ffd), np.uint64, "density_fx", C.c_uint64)
        arr("horizon", (p.ftd, p.ffd), np.uint64, "horizon_fx", C.c_uint64)
    if f64:
        arr("density_f64", (p.hd, p.ftd, p.ffd), np.float64, "density_f64", C.c_double)
        arr("horizon_f64", (p.ftd, p.ffd), np.float64, "horizon_f64", C.c_double)
    if particles:
        arr("ttime", (9, n), np.float64, "ttime", C.c_double)
        arr("fate", (n,), np.int32, "fate", C.c_int32)
        arr("steps", (n,), np.int64, "steps", C.c_int64)
    if speed_hist and p.n_speed_bins > 0:
        arr("speed_hist", (ncell, p.n_speed_bins), np.uint64, "speed_hist", C.c_uint64)
    if v_record:
        cap = 100 * p.ftd * p.hd
        arr("v_record", (cap, 3), np.float64, "v_record", C.c_double)
        arr("v_td", (cap,), np.int32, "v_td", C.c_int32)
        arr("v_fd", (cap,), np.int32, "v_fd", C.c_int32)
        arr("v_ht", (cap,), np.int32, "v_ht", C.c_int32)
        arr("v_count_nn", (p.ftd * p.hd,), np.int32, "v_count_nn", C.c_int32)
        o.v_cap = cap
    vt = vtable()
    col = _addr(collision.struct) if collision is not None else None
    rc = lib().or_run(_addr(p), _addr(surface.struct), col, C.byref(vt), rng, rr_seed,
                      pid_begin, n, nthreads, C.byref(o))
    if rc != 0:
        raise RuntimeError(f"or_run failed: {rc}")
    for k in ("total_steps", "n_escaped", "n_collisions", "n_bound_launch", "n_drift_flagged",
              "n_records"):
        res[k] = int(getattr(o, k))
    if v_record:
        k = res["n_records"]
        for name in ("v_record", "v_td", "v_fd", "v_ht"):
            res[name] = res[name][:k]
    del nh
    return res


def thermal(ftd: int, ffd: int, tp, flux: np.ndarray | None = None) -> tuple[np.ndarray, int]:
    """The oracle's thermal column model: surface temperature [ftd][ffd] and depth points."""
    F = None if flux is None else np.ascontiguousarray(flux, dtype=np.float64)
    T = np.zeros((ftd, ffd))
    h = C.c_int()
    rc = lib().or_thermal_solve(ftd, ffd, _addr(tp), _p(F) if F is not None else None, _p(T),
                                C.byref(h))
    if rc != 0:
        raise RuntimeError(f"or_thermal_solve failed: {rc}")
    return T, h.value


def reference_thermal(ftd: int, ffd: int, tp, flux: np.ndarray | None = None) -> np.ndarray | None:
    """The reference's own thermal_solve (oracle/_ref/libdsmcref.so), or None when that build is
    absent. Its stdout lines go to the process's stdout."""
    so = REF_DIR / "libdsmcref.so"
    if not so.exists():
        return None
    from dsmc_suite_b200 import _native as N
    R = C.CDLL(str(so))
    R.thermal_solve.restype = None
    R.thermal_solve.argtypes = [C.POINTER(N.SphericalGrid), C.POINTER(N.ThermalParams),
                                C.POINTER(C.c_double), C.c_int]
    T = np.zeros((ftd, ffd))
    g = N.SphericalGrid(ftd=ftd, ffd=ffd, hd=1, temperature=_p(T))
    F = None if flux is None else np.ascontiguousarray(flux, dtype=np.float64)
    R.thermal_solve(C.byref(g), C.byref(tp), _p(F) if F is not None else None, 1)
    return T


def shadow_flux(spot, facet, normal, za: float, tt: int, nmonte: int, nthreads: int = 8):
    """The oracle's Monte Carlo shadow flux F [nface][tt] (brute-force occlusion)."""
    spot = np.ascontiguousarray(spot, dtype=np.float64)
    facet = np.ascontiguousarray(facet, dtype=np.int32)
    normal = np.ascontiguousarray(normal, dtype=np.float64)
    F = np.zeros((facet.shape[0], tt))
    rc = lib().or_shadow_flux(spot.shape[0], _p(spot), facet.shape[0], _p(facet, C.c_int32),
                              _p(normal), za, tt, nmonte, _p(F), nthreads)
    if rc != 0:
        raise RuntimeError(f"or_shadow_flux failed: {rc}")
    return F


def reference_shadow_flux(spot, facet, za_deg: float, tt: int, nmonte: int, workdir,
                          nthreads: int = 8):
    """The reference's own ray tracer, run_raytracer of src/raytracer/shadow_maker.c compiled
    unmodified into oracle/_ref/libshadowref.so against the brute-force Embree stand-in of
    oracle/embree_shim/. Writes the mesh files it reads (vertices, 1-based face triples), runs it
    and returns its flux file as F [nface][tt] (printed %9.7f), or None when that build is absent."""
    from pathlib import Path
    so = REF_DIR / "libshadowref.so"
    if not so.exists():
        return None
    spot = np.ascontiguousarray(spot, dtype=np.float64)
    facet = np.ascontiguousarray(facet, dtype=np.int64)
    d = Path(workdir)
    (d / "ref_vert.txt").write_text("".join(f"{x:.17g} {y:.17g} {z:.17g}\n" for x, y, z in spot))
    (d / "ref_face.txt").write_text("".join(f"{a + 1} {b + 1} {c + 1}\n" for a, b, c in facet))
    R = C.CDLL(str(so))
    R.run_raytracer.restype = None
    R.run_raytracer.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_int,
                                C.c_int, C.c_char_p, C.c_int]
    out = d / "ref_flux.dat"
    R.run_raytracer(str(d / "ref_vert.txt").encode(), str(d / "ref_face.txt").encode(),
                    spot.shape[0], facet.shape[0], za_deg, tt, nmonte, str(out).encode(), nthreads)
    vals = out.read_text().split()
    assert int(vals[0]) == facet.shape[0] and int(vals[1]) == tt
    return np.array(vals[2:], dtype=np.float64).reshape(facet.shape[0], tt)
