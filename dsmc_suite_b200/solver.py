"""Python handle on one device context of the C ABI (include/dsmc_cuda.h).

A thin owner of a dsmc_ctx: it keeps the input arrays alive, converts results to numpy, and raises
DsmcError on any non-zero status. Every solve runs in the CUDA library; nothing here computes
particles on the host.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class Context:
    def __init__(self, device: int = 0):
        self._lib = N.lib()
        h = C.c_void_p()
        N.check(self._lib.dsmc_ctx_create(device, C.byref(h)), "dsmc_ctx_create")
        self.h = h
        self.params: N.Params | None = None
        self._keep = ()
        self._out_cap = 0

    # lifecycle --------------------------------------------------------------------------------
    def close(self) -> None:
        if self.h:
            self._lib.dsmc_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int, where: str) -> None:
        N.check(status, where, self.h)

    def set_launch_shape(self, block: int, blocks_per_sm: int, steps_per_launch: int,
                         launches_per_graph: int) -> None:
        self._check(self._lib.dsmc_set_launch_shape(self.h, block, blocks_per_sm, steps_per_launch,
                                                    launches_per_graph), "set_launch_shape")

    def launch_info(self) -> tuple[int, int]:
        """(kernel launches of the last run, resident slots) of the FAST paths."""
        la, ns = C.c_int64(), C.c_int64()
        self._check(self._lib.dsmc_get_launch_info(self.h, C.byref(la), C.byref(ns)), "launch_info")
        return la.value, ns.value

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(self._lib.dsmc_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)), "set_stream")

    # problem ----------------------------------------------------------------------------------
    def setup(self, params: N.Params, surface: N.SurfaceInputs,
              collision: N.CollisionInputs | None = None) -> None:
        col = C.byref(collision.struct) if collision is not None else None
        self._check(self._lib.dsmc_setup(self.h, C.byref(params), C.byref(surface.struct), col),
                    "dsmc_setup")
        self.params = params.copy()
        self._keep = (surface, collision)

    def enable_particle_outputs(self, n: int) -> None:
        self._check(self._lib.dsmc_enable_particle_outputs(self.h, n), "particle outputs")
        self._out_cap = n

    def zero(self) -> None:
        self._check(self._lib.dsmc_zero(self.h), "dsmc_zero")

    def run(self, path: int, pid_begin: int, n: int) -> None:
        self._check(self._lib.dsmc_run(self.h, path, pid_begin, n), "dsmc_run")

    def sync(self) -> None:
        self._check(self._lib.dsmc_sync(self.h), "dsmc_sync")

    # results ----------------------------------------------------------------------------------
    def density(self) -> np.ndarray:
        p = self.params
        out = np.zeros((p.hd, p.ftd, p.ffd), dtype=np.uint64)
        self._check(self._lib.dsmc_get_density(self.h, N.ptr(out, C.c_uint64)), "density")
        return out

    def horizon(self) -> np.ndarray:
        p = self.params
        out = np.zeros((p.ftd, p.ffd), dtype=np.uint64)
        self._check(self._lib.dsmc_get_horizon(self.h, N.ptr(out, C.c_uint64)), "horizon")
        return out

    def speed_hist(self) -> np.ndarray:
        p = self.params
        out = np.zeros((p.ncell, p.n_speed_bins), dtype=np.uint64)
        self._check(self._lib.dsmc_get_speed_hist(self.h, N.ptr(out, C.c_uint64)), "speed hist")
        return out

    def stats(self) -> dict:
        s = N.Stats()
        self._check(self._lib.dsmc_get_stats(self.h, C.byref(s)), "stats")
        return s.as_dict()

    def particle_outputs(self, n: int):
        ttime = np.zeros((9, n))
        fate = np.zeros(n, dtype=np.int32)
        steps = np.zeros(n, dtype=np.int64)
        self._check(self._lib.dsmc_get_particle_outputs(self.h, n, N.ptr(ttime),
                                                        N.ptr(fate, C.c_int32),
                                                        N.ptr(steps, C.c_int64)),
                    "particle outputs")
        return ttime, fate, steps

    def density_device(self) -> tuple[int, int]:
        p = C.POINTER(C.c_uint64)()
        n = C.c_int64()
        self._check(self._lib.dsmc_density_device(self.h, C.byref(p), C.byref(n)), "density_device")
        return C.cast(p, C.c_void_p).value or 0, n.value

    def horizon_device(self) -> tuple[int, int]:
        p = C.POINTER(C.c_uint64)()
        n = C.c_int64()
        self._check(self._lib.dsmc_horizon_device(self.h, C.byref(p), C.byref(n)), "horizon_device")
        return C.cast(p, C.c_void_p).value or 0, n.value

    # fits and records -------------------------------------------------------------------------
    def fit_samples(self, speeds: np.ndarray, counts: np.ndarray, degree: int):
        speeds = np.ascontiguousarray(speeds, dtype=np.float64)
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        ncell, mpc = speeds.shape
        coef, box = np.zeros((ncell, N.CDF_STRIDE)), np.zeros((ncell, 4))
        total, valid = np.zeros(ncell), np.zeros(ncell, dtype=np.int32)
        self._check(self._lib.dsmc_fit_cdf_samples_host(
            self.h, ncell, mpc, N.ptr(speeds), N.ptr(counts, C.c_int32), degree, N.ptr(coef),
            N.ptr(box), N.ptr(total), N.ptr(valid, C.c_int32)), "fit samples")
        return coef, box, total, valid

    def fit_hist(self, hist: np.ndarray, bin_width: float, degree: int):
        hist = np.ascontiguousarray(hist, dtype=np.uint64)
        ncell, nb = hist.shape
        coef, box = np.zeros((ncell, N.CDF_STRIDE)), np.zeros((ncell, 4))
        total, valid = np.zeros(ncell), np.zeros(ncell, dtype=np.int32)
        self._check(self._lib.dsmc_fit_cdf_hist_host(
            self.h, ncell, nb, bin_width, N.ptr(hist, C.c_uint64), degree, N.ptr(coef),
            N.ptr(box), N.ptr(total), N.ptr(valid, C.c_int32)), "fit hist")
        return coef, box, total, valid

    def push(self, path: int, pos: np.ndarray, vel: np.ndarray, nsteps: int):
        """Fed-state push of [n][3] positions/velocities (copies); returns (pos, vel, status,
        steps_taken)."""
        P = np.ascontiguousarray(pos, dtype=np.float64).copy()
        V = np.ascontiguousarray(vel, dtype=np.float64).copy()
        n = P.shape[0]
        st = np.zeros(n, dtype=np.int32)
        tk = np.zeros(n, dtype=np.int32)
        self._check(self._lib.dsmc_push_host(self.h, path, n, nsteps, N.ptr(P), N.ptr(V),
                                             N.ptr(st, C.c_int32), N.ptr(tk, C.c_int32)), "push")
        return P, V, st, tk

    def velocity_record(self, n: int, per_bucket: int = 200, total_cap: int | None = None):
        p = self.params
        if total_cap is None:
            total_cap = 100 * p.ftd * p.hd
        v = np.zeros((max(total_cap, 1), 3))
        td = np.zeros(max(total_cap, 1), dtype=np.int32)
        fd = np.zeros_like(td)
        ht = np.zeros_like(td)
        nrec = C.c_int64()
        self._check(self._lib.dsmc_velocity_record(
            self.h, n, per_bucket, total_cap, N.ptr(v), N.ptr(td, C.c_int32),
            N.ptr(fd, C.c_int32), N.ptr(ht, C.c_int32), C.byref(nrec)), "velocity record")
        k = nrec.value
        return v[:k], td[:k], fd[:k], ht[:k]

    # thermal model -----------------------------------------------------------------------------
    def thermal(self, ftd: int = 36, ffd: int = 72, tp: N.ThermalParams | None = None,
                flux: np.ndarray | None = None) -> tuple[np.ndarray, int]:
        """Surface temperature [ftd][ffd] of the thermal column model on the device, and the
        number of depth points."""
        tp = N.ThermalParams.default() if tp is None else tp
        F = None if flux is None else np.ascontiguousarray(flux, dtype=np.float64)
        T = np.zeros((ftd, ffd))
        h = C.c_int()
        self._check(self._lib.dsmc_thermal_solve_host(self.h, ftd, ffd, C.byref(tp), N.ptr(F),
                                                      N.ptr(T), C.byref(h)), "thermal")
        return T, h.value

    def last_kernel_ms(self) -> float:
        """Device time of the last thermal or shadow-flux kernel on this context."""
        ms = C.c_double()
        self._check(self._lib.dsmc_last_kernel_ms(self.h, C.byref(ms)), "last_kernel_ms")
        return ms.value

    # shadow flux ------------------------------------------------------------------------------
    def shadow_flux(self, spot: np.ndarray, facet: np.ndarray, normal: np.ndarray, za: float,
                    tt: int = 24, nmonte: int = 50) -> np.ndarray:
        """F [nface][tt] of the Monte Carlo shadow model on the device (za in radians)."""
        spot = np.ascontiguousarray(spot, dtype=np.float64)
        facet = np.ascontiguousarray(facet, dtype=np.int32)
        normal = np.ascontiguousarray(normal, dtype=np.float64)
        F = np.zeros((facet.shape[0], tt))
        self._check(self._lib.dsmc_shadow_flux_host(self.h, spot.shape[0], N.ptr(spot),
                                                    facet.shape[0], N.ptr(facet, C.c_int32),
                                                    N.ptr(normal), za, tt, nmonte, N.ptr(F)),
                    "shadow_flux")
        return F

    # one-call solve ---------------------------------------------------------------------------
    def solve(self, path: int, params: N.Params, surface: N.SurfaceInputs, n: int,
              collision: N.CollisionInputs | None = None, outputs: bool = False) -> dict:
        """Set up, solve n particles from pid 0, and return grids and statistics."""
        self.setup(params, surface, collision)
        if outputs:
            self.enable_particle_outputs(n)
        self.zero()
        self.run(path, 0, n)
        self.sync()
        res = {"density": self.density(), "horizon": self.horizon(), "stats": self.stats()}
        if outputs:
            res["ttime"], res["fate"], res["steps"] = self.particle_outputs(n)
        return res
