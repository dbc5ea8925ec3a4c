"""Shadow-flux model on the CPU: the oracle's invariants and the kept mesh entry points (no GPU).

The reference traces with Intel Embree (absent here), so the oracle's occlusion test is a
brute-force Moller-Trumbore over every triangle; its sampling and flux arithmetic follow the
reference exactly. A convex body casts no shadows, so there the flux must be the clipped
cosine of the solar incidence."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def _sun(za, tt):
    phi = ((np.arange(tt) + 0.5) / tt) * 2.0 * np.pi + np.pi
    return np.stack([np.cos(-za) * np.sin(phi), np.cos(-za) * np.cos(phi),
                     np.full(tt, np.sin(-za))], 1)


def test_convex_body_casts_no_shadow(N, O):
    from dsmc_suite_b200 import workloads as W
    spot, facet = W.cratered_mesh(3, craters=0)
    n = N.mesh_normals(spot, facet)["normal"]
    F = O.shadow_flux(spot, facet, n, 0.3, 10, 16)
    c6 = n @ _sun(0.3, 10).T
    np.testing.assert_allclose(F, np.where(c6 < 0, 0.0, c6), atol=1e-12)


def test_craters_cast_shadows_and_flux_is_bounded(N, O):
    from dsmc_suite_b200 import workloads as W
    spot, facet = W.cratered_mesh(3, depth=0.3)
    n = N.mesh_normals(spot, facet)["normal"]
    F = O.shadow_flux(spot, facet, n, 0.2, 12, 32)
    c6 = np.where(n @ _sun(0.2, 12).T < 0, 0.0, n @ _sun(0.2, 12).T)
    assert (F <= c6 + 1e-12).all() and (F >= 0).all()
    assert np.mean(F < c6 - 1e-9) > 0.01          # some lit facets are (partly) in shadow
    # the shadowed fraction is a multiple of 1 / nmonte
    lit = c6 > 1e-6
    frac = (1.0 - F[lit] / c6[lit]) * 32
    np.testing.assert_allclose(frac, np.round(frac), atol=1e-6)


def test_kept_mesh_entry_points(N, tmp_path):
    from dsmc_suite_b200 import workloads as W
    spot, facet = W.cratered_mesh(2, depth=0.2)
    (tmp_path / "v.dat").write_text("".join("%.17g %.17g %.17g\n" % tuple(p) for p in spot))
    (tmp_path / "f.dat").write_text("".join("%d %d %d\n" % tuple(f + 1) for f in facet))
    L = N.lib()
    m = L.mesh_load(str(tmp_path / "v.dat").encode(), str(tmp_path / "f.dat").encode(),
                    len(spot), len(facet))
    try:
        L.mesh_compute_normals(m)
        M = m.contents
        got = np.ctypeslib.as_array(M.face_normal, shape=(len(facet) * 3,)).reshape(-1, 3)
        a, b, c = (spot[facet[:, j]] for j in range(3))
        nrm = np.cross((c - a) / np.linalg.norm(c - a, axis=1)[:, None],
                       (b - a) / np.linalg.norm(b - a, axis=1)[:, None])
        nrm /= np.linalg.norm(nrm, axis=1)[:, None]
        nrm *= np.sign(np.einsum("ij,ij->i", nrm, (a + b + c) / 3))[:, None]
        np.testing.assert_allclose(got, nrm, atol=1e-12)
        area = np.ctypeslib.as_array(M.face_area, shape=(len(facet),))
        np.testing.assert_allclose(area, np.linalg.norm(np.cross(b - a, c - a), axis=1) / 2, rtol=1e-12)
    finally:
        L.mesh_free(m)
    # random_point_on_triangle draws rand_r twice: r1 = sqrt(u1), r2 = u2
    libc = C.CDLL("libc.so.6")
    libc.rand_r.restype = C.c_int
    libc.rand_r.argtypes = [C.POINTER(C.c_uint)]
    s1, s2 = C.c_uint(77), C.c_uint(77)
    A, B, Cv = N.Vec3(1, 0, 0), N.Vec3(0, 1, 0), N.Vec3(0, 0, 1)
    p = L.random_point_on_triangle(A, B, Cv, C.byref(s1))
    r1 = np.sqrt(libc.rand_r(C.byref(s2)) / 2147483647.0)
    r2 = libc.rand_r(C.byref(s2)) / 2147483647.0
    assert (p.x, p.y, p.z) == (1.0 - r1, r1 * (1.0 - r2), r1 * r2)
    assert s1.value == s2.value


def test_oracle_matches_the_reference_ray_tracer(N, O, tmp_path):
    """The reference's own shadow_maker.c (run_raytracer, compiled unmodified against the
    brute-force Embree stand-in of oracle/embree_shim/) pins the oracle's sampling, occlusion
    rays and flux arithmetic: its flux file equals the oracle's flux to the printed precision."""
    from dsmc_suite_b200 import workloads as W
    spot, facet = W.cratered_mesh(3, depth=0.3)
    za_deg, tt, nmonte = 17.0, 6, 16
    ref = O.reference_shadow_flux(spot, facet, za_deg, tt, nmonte, tmp_path)
    if ref is None:
        pytest.skip("oracle/_ref/libshadowref.so not built (reference sources absent)")
    n = N.mesh_normals(spot, facet)["normal"]
    F = O.shadow_flux(spot, facet, n, za_deg / 180.0 * np.pi, tt, nmonte)
    np.testing.assert_allclose(F, ref, atol=6e-8, rtol=0)
    c6 = np.where(n @ _sun(za_deg / 180.0 * np.pi, tt).T < 0, 0.0, n @ _sun(za_deg / 180.0 * np.pi, tt).T)
    assert np.mean(ref < c6 - 1e-6) > 0.01        # shadows were cast and matched
