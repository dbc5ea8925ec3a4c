"""Problem set-up for the CPU oracle - TEST INFRASTRUCTURE ONLY.

A restatement, in Python on the host, of the parameter presets and surfaces that the product
builds in C (dsmc_suite_b200/csrc/host_setup.c), so that the oracle's own runs - in particular
`bench.py --impl reference`, the timed CPU arm - build their inputs without loading the product
library. The ctypes structures mirror include/dsmc_params.h field for field; every arithmetic step
below is a double-precision IEEE operation or a libm call in the same order as the C code, so the
results are bit-identical to it (checked by tests/test_oracle_golden.py).

Sources of the constants:
  * reference model: include/constants.h:5-35 and the runner fills of src/dsmc/ballistic.c:49-67
    and src/dsmc/advanced.c:131-152 of the reference;
  * config model: the benchmark workloads (Ceres-like body, H2O, dt 2 s, 20,000-step lives,
    50 exponential shells to 10 R x 36 x 72, photolysis lifetime 2.6e5 s).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

MODEL_REFERENCE, MODEL_CONFIG = 0, 1
RUNNER_BALLISTIC, RUNNER_ADVANCED = 0, 1
SCATTER_REFERENCE, SCATTER_ISOTROPIC = 0, 1


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

    @property
    def ncell(self) -> int:
        return self.hd * self.ftd * self.ffd


class Surface(C.Structure):
    """dsmc_surface (include/dsmc_params.h)."""
    _fields_ = [
        ("T_map", C.POINTER(C.c_double)), ("nface", C.c_int32), ("nlevel", C.c_int32),
        ("face_verts", C.POINTER(C.c_double)), ("face_T", C.POINTER(C.c_double)),
        ("face_cdf", C.POINTER(C.c_double)), ("base_centroid", C.POINTER(C.c_double)),
        ("split_planes", C.POINTER(C.c_double)),
    ]


def _dp(a: np.ndarray | None):
    return C.POINTER(C.c_double)() if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


# reference constants (include/constants.h:5-35 of the reference)
_G, _M_CERES, _R_CERES = 6.67e-11, 9.39e20, 476.2e3
_K_B, _MOLE, _MMASS = 1.38e-23, 6.02e23, 18e-3
_P_CERES = 9.07417 * 3600.0
_LIFETIME = 1.0 / 1.02e-5 * (2.8 * 2.8)


def params_reference(runner: int, ftd: int = 36, ffd: int = 72) -> Params:
    """The reference runners' parameter fills (ballistic.c:49-67, advanced.c:131-152)."""
    p = Params()
    p.model, p.runner, p.ftd, p.ffd = MODEL_REFERENCE, runner, ftd, ffd
    p.GM = _G * _M_CERES
    p.Radii = _R_CERES
    p.ve = math.sqrt(2.0 * _G * _M_CERES / _R_CERES)
    p.lifetime = _LIFETIME
    p.P = _P_CERES
    p.alpha = 0.5
    p.dt_rot = p.P / ffd
    p.kB_over_m = _K_B / (_MMASS / _MOLE)
    p.freeze_T, p.w_min = 100.0, 0.01
    p.hop_step_cap, p.life_step_cap = 10000000, 0
    p.drift_tol = 1e-2
    p.scatter = SCATTER_REFERENCE
    p.seed = 20261203
    if runner == RUNNER_BALLISTIC:
        p.dt_step, p.use_exp_grid = 5.0, 0
        p.unih = p.Radii * 0.1
        p.alpha2, p.hd = 0.0, 100
        p.max_height = p.unih * p.hd + p.Radii
        p.skip_first_deposit, p.collide_ht_max = 1, 0
    elif runner == RUNNER_ADVANCED:
        p.dt_step, p.cross_section, p.use_exp_grid, p.hd = 0.5, 1e-19, 1, 50
        p.max_height = 3e6 * math.sqrt(2.0)
        p.alpha2 = 0.04
        p.unih = (p.max_height - p.Radii) / (math.pow(1.0 + p.alpha2, p.hd) - 1.0) * p.alpha2
        p.skip_first_deposit, p.collide_ht_max = 1, p.hd // 3
    else:
        raise ValueError("runner must be RUNNER_BALLISTIC or RUNNER_ADVANCED")
    p.log1p_alpha2 = math.log(1.0 + p.alpha2)
    p.wdecay = math.exp(-p.dt_step / p.lifetime)
    return p


def params_config(runner: int = RUNNER_BALLISTIC, Radii: float = 470e3, GM: float = 6.26e10,
                  hd: int = 50, seed: int = 20261203) -> Params:
    """The config-model parameters of the benchmark workloads."""
    if Radii <= 0.0 or GM <= 0.0 or hd < 1 or runner not in (RUNNER_BALLISTIC, RUNNER_ADVANCED):
        raise ValueError("invalid config-model parameters")
    k_B, m, d = 1.380649e-23, 2.99e-26, 4.6e-10
    p = Params()
    p.model, p.runner, p.ftd, p.ffd, p.hd, p.use_exp_grid = MODEL_CONFIG, runner, 36, 72, hd, 1
    p.GM, p.Radii = GM, Radii
    p.ve = math.sqrt(2.0 * GM / Radii)
    p.lifetime, p.P, p.dt_step = 2.6e5, _P_CERES, 2.0
    p.dt_rot = p.P / p.ffd
    p.max_height = 10.0 * Radii
    p.alpha2 = 0.04
    p.unih = (p.max_height - Radii) / (math.pow(1.0 + p.alpha2, hd) - 1.0) * p.alpha2
    p.log1p_alpha2 = math.log(1.0 + p.alpha2)
    p.wdecay = math.exp(-p.dt_step / p.lifetime)
    p.alpha = 1.0
    p.cross_section = math.pi * d * d
    p.kB_over_m = k_B / m
    p.freeze_T, p.w_min = 0.0, 0.01
    p.sun[0] = 1.0
    p.hop_step_cap, p.life_step_cap = 20000, 20000
    p.skip_first_deposit, p.scatter, p.collide_ht_max = 0, SCATTER_ISOTROPIC, hd
    p.redraw_col_threshold = 1
    p.seed = seed
    p.n_speed_bins, p.speed_bin_width = 0, 25.0
    p.drift_tol = 1e-2
    return p


# ------------------------------------------------------------------------------------------
# Icosphere: midpoint subdivision of the icosahedron, faces in subdivision order.

def _norm(v):
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return [v[0] / n, v[1] / n, v[2] / n]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


class Icosphere:
    """Face vertices [nface][9], base-face centroids [20][3] and the corner-cut planes
    [nnode][9] of every parent face (children 0, 1, 2 at the corners a, b, c, 3 the centre)."""

    def __init__(self, nlevel: int = 3):
        if not 0 <= nlevel <= 6:
            raise ValueError("nlevel must lie in [0, 6]")
        self.nlevel = nlevel
        self.nface = 20 << (2 * nlevel)
        self.nnode = 20 * ((1 << (2 * nlevel)) - 1) // 3
        self.face_verts = np.zeros((self.nface, 9))
        self.base_centroid = np.zeros((20, 3))
        self.split_planes = np.zeros((max(self.nnode, 1), 9))
        t = (1.0 + math.sqrt(5.0)) / 2.0
        V = []
        for perm in range(3):
            for s1 in (-1, 1):
                for s2 in (-1, 1):
                    q = [0.0, s1 * 1.0, s2 * t]
                    V.append([q[(3 - perm) % 3], q[(4 - perm) % 3], q[(5 - perm) % 3]])
        nf = 0
        for i in range(12):
            for j in range(i + 1, 12):
                for k in range(j + 1, 12):
                    d = [sum((V[x][c] - V[y][c]) * (V[x][c] - V[y][c]) for c in range(3))
                         for x, y in ((i, j), (j, k), (k, i))]
                    if any(abs(e - 4.0) > 1e-9 for e in d):
                        continue
                    a, b, c = list(V[i]), list(V[j]), list(V[k])
                    e1 = [b[x] - a[x] for x in range(3)]
                    e2 = [c[x] - a[x] for x in range(3)]
                    s = [a[x] + b[x] + c[x] for x in range(3)]
                    if _dot(_cross(e1, e2), s) < 0.0:
                        b, c = c, b
                    a, b, c = _norm(a), _norm(b), _norm(c)
                    self.base_centroid[nf] = _norm([a[x] + b[x] + c[x] for x in range(3)])
                    self._subdivide(a, b, c, 0, nf)
                    nf += 1
        if nf != 20:
            raise RuntimeError("icosahedron construction failed")

    def _subdivide(self, a, b, c, level, node):
        if level == self.nlevel:
            self.face_verts[node] = a + b + c
            return
        ab = _norm([0.5 * (a[k] + b[k]) for k in range(3)])
        bc = _norm([0.5 * (b[k] + c[k]) for k in range(3)])
        ca = _norm([0.5 * (c[k] + a[k]) for k in range(3)])
        off = 20 * ((1 << (2 * level)) - 1) // 3
        for k, (corner, p0, p1) in enumerate(((a, ab, ca), (b, bc, ab), (c, ca, bc))):
            n = _cross(p0, p1)
            if _dot(n, corner) < 0.0:
                n = [-n[0], -n[1], -n[2]]
            self.split_planes[off + node, 3 * k:3 * k + 3] = n
        self._subdivide(a, ab, ca, level + 1, node * 4 + 0)
        self._subdivide(b, bc, ab, level + 1, node * 4 + 1)
        self._subdivide(c, ca, bc, level + 1, node * 4 + 2)
        self._subdivide(ab, bc, ca, level + 1, node * 4 + 3)

    def face_temperature(self, sun=(1.0, 0.0, 0.0), T_ss: float = 235.0,
                         T_floor: float = 110.0) -> np.ndarray:
        """T = max(T_floor, T_ss cos(z)^(1/4)) at each face centroid."""
        out = np.zeros(self.nface)
        for f in range(self.nface):
            v = self.face_verts[f].tolist()
            cz = _dot(_norm([v[0] + v[3] + v[6], v[1] + v[4] + v[7], v[2] + v[5] + v[8]]),
                      [float(x) for x in sun])
            T = T_ss * math.pow(cz, 0.25) if cz > 0.0 else 0.0
            out[f] = T if T > T_floor else T_floor
        return out


def latlon_temperature(ftd: int = 36, ffd: int = 72, sun=(1.0, 0.0, 0.0), T_ss: float = 235.0,
                       T_floor: float = 110.0) -> np.ndarray:
    """The same formula at the latitude-longitude cell centres, positions in the reference's
    convention (cos th sin fi, cos th cos fi, sin th) of ballistic.c:114-118."""
    T = np.zeros((ftd, ffd))
    s = [float(x) for x in sun]
    for td in range(ftd):
        th = (td + 0.5) / ftd * math.pi - math.pi / 2.0
        for fd in range(ffd):
            fi = (fd + 0.5) / ffd * 2.0 * math.pi
            cz = _dot([math.cos(th) * math.sin(fi), math.cos(th) * math.cos(fi), math.sin(th)], s)
            t = T_ss * math.pow(cz, 0.25) if cz > 0.0 else 0.0
            T[td, fd] = t if t > T_floor else T_floor
    return T


class SurfaceInputs:
    """Owns the arrays behind one dsmc_surface (latitude-longitude map or icosphere)."""

    def __init__(self, T_map: np.ndarray | None = None, ico: Icosphere | None = None,
                 face_T: np.ndarray | None = None, face_cdf: np.ndarray | None = None):
        self.T_map = None if T_map is None else np.ascontiguousarray(T_map, dtype=np.float64)
        self.ico = ico
        self.face_T = None if face_T is None else np.ascontiguousarray(face_T, dtype=np.float64)
        self.face_cdf = None if face_cdf is None else np.ascontiguousarray(face_cdf,
                                                                           dtype=np.float64)
        s = Surface()
        s.T_map = _dp(self.T_map)
        if ico is not None:
            s.nface, s.nlevel = ico.nface, ico.nlevel
            s.face_verts, s.base_centroid = _dp(ico.face_verts), _dp(ico.base_centroid)
            s.split_planes = _dp(ico.split_planes)
        s.face_T, s.face_cdf = _dp(self.face_T), _dp(self.face_cdf)
        self.struct = s
