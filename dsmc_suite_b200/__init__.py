"""dsmc_suite_b200 - the test-particle DSMC hot path of dsmc_suite on NVIDIA B200 (sm_100a).

Host-side mirror of the reference interface:
    run_ballistic(totaln, temp_file, output_prefix, nthreads)      (src/dsmc/ballistic.c:35-36)
    run_advanced(totaln, temp_file, prev_den_file, prev_v_record_file, output_prefix, nthreads)
                                                                    (src/dsmc/advanced.c:119-121)
Both call the C runners of libdsmc_b200.so, which solve on the GPU and write the reference's
.dat files. Context (solver.py) exposes the C ABI of include/dsmc_cuda.h directly.
"""
from __future__ import annotations

from . import _native
from ._native import (DsmcError, Icosphere, SurfaceInputs, CollisionInputs, params_config,
                      params_reference, latlon_temperature, MODEL_REFERENCE, MODEL_CONFIG,
                      RUNNER_BALLISTIC, RUNNER_ADVANCED, PATH_PLAIN_FP64, PATH_FAST_FP32,
                      PATH_FAST_FP64, FIXED_SCALE)
from .solver import Context
from .server import BudgetExceeded, Server

__all__ = ["Context", "Server", "BudgetExceeded", "DsmcError", "Icosphere", "SurfaceInputs", "CollisionInputs",
           "params_config", "params_reference", "latlon_temperature", "run_ballistic",
           "run_advanced", "MODEL_REFERENCE", "MODEL_CONFIG", "RUNNER_BALLISTIC",
           "RUNNER_ADVANCED", "PATH_PLAIN_FP64", "PATH_FAST_FP32", "PATH_FAST_FP64",
           "FIXED_SCALE"]


def _cstr(s):
    return None if s is None else str(s).encode()


def run_ballistic(totaln: int, temp_file: str, output_prefix: str, nthreads: int = 1) -> None:
    """Ballistic phase on the GPU; writes <prefix>_den/_horizon/_v_record/_ttime.dat."""
    import ctypes as C
    f = _native.lib().run_ballistic
    f.restype = None
    f.argtypes = [C.c_int, C.c_char_p, C.c_char_p, C.c_int]
    f(int(totaln), _cstr(temp_file), _cstr(output_prefix), int(nthreads))


def run_advanced(totaln: int, temp_file: str, prev_den_file: str | None,
                 prev_v_record_file: str | None, output_prefix: str, nthreads: int = 1) -> None:
    """Collisional phase on the GPU; writes <prefix>_den/_horizon/_ttime.dat."""
    import ctypes as C
    f = _native.lib().run_advanced
    f.restype = None
    f.argtypes = [C.c_int, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
    f(int(totaln), _cstr(temp_file), _cstr(prev_den_file), _cstr(prev_v_record_file),
      _cstr(output_prefix), int(nthreads))
