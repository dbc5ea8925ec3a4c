"""ctypes view of the C ABI in include/dsmc_cuda.h and include/dsmc_params.h.

The shared library is built in-tree (dsmc_suite_b200/libdsmc_b200.so, see build.py). Loading it
needs no GPU; device calls fail with DSMC_ERR_NO_DEVICE when no CUDA device is present. There is
no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libdsmc_b200.so"

MODEL_REFERENCE, MODEL_CONFIG = 0, 1
RUNNER_BALLISTIC, RUNNER_ADVANCED = 0, 1
SCATTER_REFERENCE, SCATTER_ISOTROPIC = 0, 1
PATH_PLAIN_FP64, PATH_FAST_FP32, PATH_FAST_FP64 = 0, 1, 2
FATE_ALIVE, FATE_PHOTOLYSED, FATE_ESCAPED, FATE_FROZEN, FATE_STEP_CAP = range(5)
FIXED_SCALE = 16777216.0
VOLUME_PHYSICAL, VOLUME_REFERENCE = 0, 1
CDF_STRIDE = 8
CDF_MAX_DEGREE = 6

STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "no CUDA device",
          -4: "out of memory", -5: "call out of order", -6: "memory budget exceeded",
          -7: "file I/O error"}


class Params(C.Structure):
    """dsmc_params (include/dsmc_params.h)."""
    _fields_ = [
        ("model", C.c_int32), ("runner", C.c_int32),
        ("ftd", C.c_int32), ("ffd", C.c_int32), ("hd", C.c_int32),
        ("use_exp_grid", C.c_int32),
        ("GM", C.c_double), ("Radii", C.c_double), ("ve", C.c_double),
        ("lifetime", C.c_double), ("P", C.c_double), ("dt_step", C.c_double),
        ("dt_rot", C.c_double), ("max_height", C.c_double), ("unih", C.c_double),
        ("alpha2", C.c_double), ("log1p_alpha2", C.c_double), ("wdecay", C.c_double),
        ("alpha", C.c_double), ("cross_section", C.c_double), ("kB_over_m", C.c_double),
        ("freeze_T", C.c_double), ("w_min", C.c_double), ("sun", C.c_double * 3),
        ("hop_step_cap", C.c_int64), ("life_step_cap", C.c_int64),
        ("skip_first_deposit", C.c_int32), ("scatter", C.c_int32),
        ("collide_ht_max", C.c_int32), ("redraw_col_threshold", C.c_int32),
        ("seed", C.c_uint64), ("instance", C.c_uint32), ("n_speed_bins", C.c_int32),
        ("speed_bin_width", C.c_double), ("drift_tol", C.c_double),
    ]

    def copy(self) -> "Params":
        out = Params()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(Params))
        return out

    @property
    def ncell(self) -> int:
        return self.hd * self.ftd * self.ffd


class Surface(C.Structure):
    """dsmc_surface."""
    _fields_ = [
        ("T_map", C.POINTER(C.c_double)), ("nface", C.c_int32), ("nlevel", C.c_int32),
        ("face_verts", C.POINTER(C.c_double)), ("face_T", C.POINTER(C.c_double)),
        ("face_cdf", C.POINTER(C.c_double)), ("base_centroid", C.POINTER(C.c_double)),
        ("split_planes", C.POINTER(C.c_double)),
    ]


class Collision(C.Structure):
    """dsmc_collision."""
    _fields_ = [
        ("n_bg", C.POINTER(C.c_double)), ("n_bg_len", C.c_int64),
        ("cdf_coef", C.POINTER(C.c_double)), ("cdf_box", C.POINTER(C.c_double)),
        ("cdf_total", C.POINTER(C.c_double)), ("cdf_valid", C.POINTER(C.c_int32)),
        ("cdf_degree", C.c_int32),
    ]


class Stats(C.Structure):
    """dsmc_stats."""
    _fields_ = [(n, C.c_int64) for n in ("total_steps", "n_escaped", "n_collisions",
                                          "n_bound_launch", "n_finished", "n_drift_flagged")]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class ThermalParams(C.Structure):
    """ThermalParams (include/thermal.h, the reference's layout)."""
    _fields_ = [("density", C.c_double), ("conductivity", C.c_double), ("Cp", C.c_double),
                ("albedo", C.c_double), ("distance_AU", C.c_double), ("depth", C.c_double),
                ("n_substep", C.c_int), ("z_angle", C.c_double), ("p_mat", C.c_double * 5),
                ("LH_mat", C.c_double * 5), ("tran_unit_p", C.c_double),
                ("tran_unit_LH", C.c_double)]

    @staticmethod
    def default() -> "ThermalParams":
        tp = ThermalParams()
        lib().thermal_params_default(C.byref(tp))
        return tp


class SphericalGrid(C.Structure):
    """SphericalGrid (include/types.h, the reference's layout)."""
    _fields_ = [("ftd", C.c_int), ("ffd", C.c_int), ("hd", C.c_int),
                ("density", C.POINTER(C.c_double)), ("temperature", C.POINTER(C.c_double)),
                ("volume", C.POINTER(C.c_double)), ("horizon", C.POINTER(C.c_double))]


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class Mesh(C.Structure):
    """Mesh (include/types.h, the reference's layout)."""
    _fields_ = [("npoint", C.c_int), ("nface", C.c_int), ("spot", C.POINTER(C.c_double)),
                ("facet", C.POINTER(C.c_int)), ("face_normal", C.POINTER(C.c_double)),
                ("face_area", C.POINTER(C.c_double)), ("loc_xyz", C.POINTER(C.c_double)),
                ("dir", C.POINTER(C.c_double))]


def mesh_normals(spot: np.ndarray, facet: np.ndarray) -> dict:
    """The kept mesh_compute_normals on numpy arrays: spot [npoint][3], facet [nface][3] 0-based.
    Returns normals, areas, centroids and (latitude, longitude) directions."""
    spot = np.ascontiguousarray(spot, dtype=np.float64)
    facet = np.ascontiguousarray(facet, dtype=np.int32)
    nf = facet.shape[0]
    out = {"normal": np.zeros((nf, 3)), "area": np.zeros(nf), "centroid": np.zeros((nf, 3)),
           "dir": np.zeros((nf, 2))}
    m = Mesh(npoint=spot.shape[0], nface=nf, spot=ptr(spot), facet=ptr(facet, C.c_int),
             face_normal=ptr(out["normal"]), face_area=ptr(out["area"]),
             loc_xyz=ptr(out["centroid"]), dir=ptr(out["dir"]))
    lib().mesh_compute_normals(C.byref(m))
    return out


class ServerInfo(C.Structure):
    """dsmc_server_info."""
    _fields_ = [(n, C.c_int64) for n in ("submitted", "completed", "fetched", "rejected", "active",
                                          "bytes_in_use", "bytes_budget", "slots", "rounds",
                                          "launches", "total_steps")] + [("busy_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class RequestInfo(C.Structure):
    """dsmc_request_info."""
    _fields_ = [("n", C.c_int64), ("ncell", C.c_int64), ("nhcell", C.c_int64),
                ("t_submit", C.c_double), ("t_done", C.c_double)]


def ptr(a: np.ndarray | None, ctype=C.c_double):
    """Pointer to a contiguous numpy array (or NULL)."""
    if a is None:
        return C.POINTER(ctype)()
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_U64P = C.POINTER(C.c_uint64)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)

# (name, restype, argtypes) of every function include/dsmc_cuda.h declares.
SIGNATURES = [
    ("dsmc_params_reference", C.c_int, [C.POINTER(Params), C.c_int, C.c_int, C.c_int]),
    ("dsmc_params_config", C.c_int, [C.POINTER(Params), C.c_int, C.c_double, C.c_double, C.c_int,
                                     C.c_uint64]),
    ("dsmc_icosphere_nface", C.c_int, [C.c_int]),
    ("dsmc_icosphere_nnode", C.c_int, [C.c_int]),
    ("dsmc_icosphere_build", C.c_int, [C.c_int, _DP, _DP, _DP]),
    ("dsmc_icosphere_locate", C.c_int, [C.c_int, _DP, _DP, _DP]),
    ("dsmc_face_temperature", C.c_int, [C.c_int, _DP, _DP, C.c_double, C.c_double, _DP]),
    ("dsmc_latlon_temperature", C.c_int, [C.c_int, C.c_int, _DP, C.c_double, C.c_double, _DP]),
    ("dsmc_sublimation_flux", C.c_double, [C.c_double, C.c_double]),
    ("dsmc_source_cdf", C.c_int, [C.c_int, _DP, _DP, C.c_double, _DP, _DP]),
    ("dsmc_status_string", C.c_char_p, [C.c_int]),
    ("dsmc_last_error", C.c_char_p, [_P]),
    ("dsmc_ctx_create", C.c_int, [C.c_int, C.POINTER(_P)]),
    ("dsmc_ctx_destroy", C.c_int, [_P]),
    ("dsmc_ctx_set_stream", C.c_int, [_P, _P]),
    ("dsmc_setup", C.c_int, [_P, C.POINTER(Params), C.POINTER(Surface), C.POINTER(Collision)]),
    ("dsmc_enable_particle_outputs", C.c_int, [_P, C.c_int64]),
    ("dsmc_zero", C.c_int, [_P]),
    ("dsmc_run", C.c_int, [_P, C.c_int, C.c_int64, C.c_int64]),
    ("dsmc_sync", C.c_int, [_P]),
    ("dsmc_get_density", C.c_int, [_P, _U64P]),
    ("dsmc_get_horizon", C.c_int, [_P, _U64P]),
    ("dsmc_get_stats", C.c_int, [_P, C.POINTER(Stats)]),
    ("dsmc_get_speed_hist", C.c_int, [_P, _U64P]),
    ("dsmc_get_particle_outputs", C.c_int, [_P, C.c_int64, _DP, _I32P, _I64P]),
    ("dsmc_density_device", C.c_int, [_P, C.POINTER(_U64P), _I64P]),
    ("dsmc_horizon_device", C.c_int, [_P, C.POINTER(_U64P), _I64P]),
    ("dsmc_fit_cdf_samples_host", C.c_int, [_P, C.c_int64, C.c_int, _DP, _I32P, C.c_int, _DP, _DP,
                                            _DP, _I32P]),
    ("dsmc_fit_cdf_hist_host", C.c_int, [_P, C.c_int64, C.c_int, C.c_double, _U64P, C.c_int, _DP,
                                         _DP, _DP, _I32P]),
    ("dsmc_set_launch_shape", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("dsmc_get_launch_info", C.c_int, [_P, _I64P, _I64P]),
    ("dsmc_measure_fma_peak", C.c_int, [_P, C.c_int, _DP]),
    ("dsmc_copy_grids_device", C.c_int, [_P, _U64P, _U64P]),
    ("dsmc_push_host", C.c_int, [_P, C.c_int, C.c_int64, C.c_int, _DP, _DP, _I32P, _I32P]),
    ("dsmc_velocity_record", C.c_int, [_P, C.c_int64, C.c_int, C.c_int64, _DP, _I32P, _I32P, _I32P,
                                       _I64P]),
    ("dsmc_solve_fast_noalloc", C.c_int, [C.POINTER(Params), C.POINTER(Surface), C.c_int64,
                                          C.c_int64, _U64P, _U64P, _U64P, _P]),
    ("dsmc_noalloc_last_error", C.c_char_p, []),
    ("dsmc_thermal_solve_host", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(ThermalParams), _DP,
                                          _DP, C.POINTER(C.c_int)]),
    ("thermal_params_default", None, [C.POINTER(ThermalParams)]),
    ("thermal_solve", None, [C.POINTER(SphericalGrid), C.POINTER(ThermalParams), _DP, C.c_int]),
    ("dsmc_last_kernel_ms", C.c_int, [_P, _DP]),
    ("dsmc_shadow_flux_host", C.c_int, [_P, C.c_int, _DP, C.c_int, _I32P, _DP, C.c_double,
                                        C.c_int, C.c_int, _DP]),
    ("mesh_load", C.POINTER(Mesh), [C.c_char_p, C.c_char_p, C.c_int, C.c_int]),
    ("mesh_free", None, [C.POINTER(Mesh)]),
    ("mesh_compute_normals", None, [C.POINTER(Mesh)]),
    ("random_point_on_triangle", Vec3, [Vec3, Vec3, Vec3, C.POINTER(C.c_uint)]),
    ("run_raytracer", None, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_int,
                             C.c_int, C.c_char_p, C.c_int]),
    ("dsmc_server_create", C.c_int, [C.c_int, C.c_int64, C.c_int, C.POINTER(_P)]),
    ("dsmc_server_destroy", C.c_int, [_P]),
    ("dsmc_server_last_error", C.c_char_p, [_P]),
    ("dsmc_server_set_shape", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("dsmc_server_submit", C.c_int, [_P, C.POINTER(Params), C.POINTER(Surface),
                                     C.POINTER(Collision), C.c_int64, _I64P]),
    ("dsmc_server_poll", C.c_int, [_P, _I64P, C.c_int, C.POINTER(C.c_int)]),
    ("dsmc_server_fetch", C.c_int, [_P, C.c_int64, _U64P, _U64P, C.POINTER(Stats),
                                    C.POINTER(RequestInfo)]),
    ("dsmc_server_info_get", C.c_int, [_P, C.POINTER(ServerInfo)]),
    ("dsmc_server_now", C.c_double, [_P]),
    ("dsmc_cell_volumes", C.c_int, [C.POINTER(Params), C.c_int, _DP]),
    ("dsmc_number_density_host", C.c_int, [C.POINTER(Params), _U64P, C.c_int64, C.c_double,
                                           C.c_int, _DP]),
    ("dsmc_solve_host", C.c_int, [_P, C.c_int, C.POINTER(Params), C.POINTER(Surface),
                                  C.POINTER(Collision), C.c_int64, _U64P, _U64P, C.POINTER(Stats)]),
]

_lib = None


def lib() -> C.CDLL:
    """Load libdsmc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m dsmc_suite_b200.build")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class DsmcError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)}" + (f" ({detail})" if detail else ""))


def check(status: int, where: str, ctx=None) -> None:
    if status != 0:
        detail = lib().dsmc_last_error(ctx)
        raise DsmcError(status, where, detail.decode() if detail else "")


# ----------------------------------------------------------------------------------------------
# Host-side helpers


def params_reference(runner: int, ftd: int = 36, ffd: int = 72) -> Params:
    p = Params()
    check(lib().dsmc_params_reference(C.byref(p), runner, ftd, ffd), "dsmc_params_reference")
    return p


def params_config(runner: int = RUNNER_BALLISTIC, Radii: float = 470e3, GM: float = 6.26e10,
                  hd: int = 50, seed: int = 20261203) -> Params:
    p = Params()
    check(lib().dsmc_params_config(C.byref(p), runner, Radii, GM, hd, seed), "dsmc_params_config")
    return p


class Icosphere:
    """Icosphere surface arrays (keeps the numpy buffers alive for the Surface struct)."""

    def __init__(self, nlevel: int = 3):
        L = lib()
        self.nlevel = nlevel
        self.nface = L.dsmc_icosphere_nface(nlevel)
        self.nnode = L.dsmc_icosphere_nnode(nlevel)
        self.face_verts = np.zeros((self.nface, 9))
        self.base_centroid = np.zeros((20, 3))
        self.split_planes = np.zeros((max(self.nnode, 1), 9))
        check(L.dsmc_icosphere_build(nlevel, ptr(self.face_verts), ptr(self.base_centroid),
                                     ptr(self.split_planes)), "dsmc_icosphere_build")

    def locate(self, p) -> int:
        q = np.ascontiguousarray(p, dtype=np.float64)
        return lib().dsmc_icosphere_locate(self.nlevel, ptr(self.base_centroid),
                                           ptr(self.split_planes), ptr(q))

    def face_temperature(self, sun=(1.0, 0.0, 0.0), T_ss: float = 235.0,
                         T_floor: float = 110.0) -> np.ndarray:
        T = np.zeros(self.nface)
        s = np.ascontiguousarray(sun, dtype=np.float64)
        check(lib().dsmc_face_temperature(self.nface, ptr(self.face_verts), ptr(s), T_ss, T_floor,
                                          ptr(T)), "dsmc_face_temperature")
        return T

    def source_cdf(self, face_T: np.ndarray, mmass_kg: float = 2.99e-26):
        cdf = np.zeros(self.nface)
        rate = C.c_double()
        check(lib().dsmc_source_cdf(self.nface, ptr(self.face_verts), ptr(face_T), mmass_kg,
                                    ptr(cdf), C.byref(rate)), "dsmc_source_cdf")
        return cdf, rate.value


def latlon_temperature(ftd: int = 36, ffd: int = 72, sun=(1.0, 0.0, 0.0), T_ss: float = 235.0,
                       T_floor: float = 110.0) -> np.ndarray:
    T = np.zeros((ftd, ffd))
    s = np.ascontiguousarray(sun, dtype=np.float64)
    check(lib().dsmc_latlon_temperature(ftd, ffd, ptr(s), T_ss, T_floor, ptr(T)),
          "dsmc_latlon_temperature")
    return T


def cell_volumes(p: Params, volume_mode: int = VOLUME_PHYSICAL) -> np.ndarray:
    """Cell volumes [hd][ftd][ffd] [m^3] (dsmc_cell_volumes)."""
    v = np.zeros((p.hd, p.ftd, p.ffd))
    check(lib().dsmc_cell_volumes(C.byref(p), volume_mode, ptr(v)), "dsmc_cell_volumes")
    return v


def number_density(p: Params, density_fx: np.ndarray, n: int, production_rate: float,
                   volume_mode: int = VOLUME_PHYSICAL) -> np.ndarray:
    """FP64 number density [m^-3] of a solve's fixed-point grid (dsmc_number_density_host)."""
    fx = np.ascontiguousarray(density_fx, dtype=np.uint64)
    out = np.zeros((p.hd, p.ftd, p.ffd))
    check(lib().dsmc_number_density_host(C.byref(p), ptr(fx, C.c_uint64), n, production_rate,
                                         volume_mode, ptr(out)), "dsmc_number_density_host")
    return out


class SurfaceInputs:
    """Owns the arrays behind one dsmc_surface."""

    def __init__(self, T_map: np.ndarray | None = None, ico: Icosphere | None = None,
                 face_T: np.ndarray | None = None, face_cdf: np.ndarray | None = None):
        self.T_map = None if T_map is None else np.ascontiguousarray(T_map, dtype=np.float64)
        self.ico = ico
        self.face_T = None if face_T is None else np.ascontiguousarray(face_T, dtype=np.float64)
        self.face_cdf = None if face_cdf is None else np.ascontiguousarray(face_cdf, dtype=np.float64)
        s = Surface()
        s.T_map = ptr(self.T_map)
        if ico is not None:
            s.nface, s.nlevel = ico.nface, ico.nlevel
            s.face_verts = ptr(ico.face_verts)
            s.base_centroid = ptr(ico.base_centroid)
            s.split_planes = ptr(ico.split_planes)
        s.face_T = ptr(self.face_T)
        s.face_cdf = ptr(self.face_cdf)
        self.struct = s


class CollisionInputs:
    """Owns the arrays behind one dsmc_collision."""

    def __init__(self, n_bg: np.ndarray | None, coef: np.ndarray, box: np.ndarray,
                 total: np.ndarray, valid: np.ndarray, degree: int):
        self.n_bg = None if n_bg is None else np.ascontiguousarray(n_bg, dtype=np.float64).ravel()
        self.coef = np.ascontiguousarray(coef, dtype=np.float64)
        self.box = np.ascontiguousarray(box, dtype=np.float64)
        self.total = np.ascontiguousarray(total, dtype=np.float64)
        self.valid = np.ascontiguousarray(valid, dtype=np.int32)
        c = Collision()
        c.n_bg = ptr(self.n_bg)
        c.n_bg_len = 0 if self.n_bg is None else self.n_bg.size
        c.cdf_coef, c.cdf_box, c.cdf_total = ptr(self.coef), ptr(self.box), ptr(self.total)
        c.cdf_valid = ptr(self.valid, C.c_int32)
        c.cdf_degree = degree
        self.struct = c
