"""Build the DSMC library and CLI in-tree for sm_100a.

    python -m dsmc_suite_b200.build          # or dsmc_suite_b200.build.build()

Outputs (git-ignored, shipped with the source tree):
    dsmc_suite_b200/libdsmc_b200.so   the C ABI of include/dsmc_cuda.h plus the reference's kept
                                      scalar entry points and drop-in runners
    dsmc_suite_b200/bin/dsmc_suite    the CLI (dsmc, dsmc-adv, pipeline subcommands)

CUDA sources compile with nvcc for `-gencode arch=compute_100a,code=sm_100a` only. The plain FP64
kernel's translation unit adds -fmad=false so its double arithmetic rounds every operation as the
reference's x86-64 build does. Host C compiles with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INC = ROOT / "include"
OBJ = PKG / "_build"
LIB = PKG / "libdsmc_b200.so"
CLI = PKG / "bin" / "dsmc_suite"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", f"-I{INC}", f"-I{CSRC}"] + ARCH
# per-file extra flags
CUDA_SOURCES = {
    "kernel_plain.cu": ["-fmad=false"],
    "kernel_fit.cu": ["-fmad=false"],
    "kernel_thermal.cu": ["-fmad=false"],
    "kernel_raytrace.cu": ["-fmad=false"],
    # FP32 subnormals flushed to zero: the FAST engines' FP32 values (positions, velocities and
    # their two-sum low words, weights above the photolysis cutoff, cell-test products) are far
    # from the subnormal range, and the per-step reciprocal square root then needs no subnormal
    # guard. Grids of the config workloads are bit-identical to the build without the flag; the
    # reference model's FP32 event maps (asinf, atan2f, sincosf) change at the last place. The
    # Ceres-like workload runs 2.23e11 particle-steps/s against 2.09e11 without it.
    "fast_engine.cu": ["-ftz=true"],
    "kernel_peak.cu": [],
    "noalloc.cu": [],
    "problem.cu": [],
    "server.cu": [],
    "dsmc_abi.cu": [],
}
C_SOURCES = ["host_setup.c", "host_scalar.c", "host_fileio.c", "host_runners.c", "host_thermal.c",
             "host_raytrace.c", "host_density.c"]
C_FLAGS = ["-O2", "-std=gnu11", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
           "-Wno-unused-parameter", f"-I{INC}", f"-I{CSRC}"]


def _tool(name: str) -> str:
    cand = {"nvcc": ["/usr/local/cuda/bin/nvcc"], "gcc": ["/usr/bin/gcc"]}.get(name, [])
    for c in cand:
        if os.path.exists(c):
            return c
    found = shutil.which(name)
    if not found:
        raise RuntimeError(f"{name} not found")
    return found


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every CUDA and C source, link the shared library and the CLI. Incremental."""
    OBJ.mkdir(exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    nvcc, gcc = _tool("nvcc"), _tool("gcc")
    # objects depend on the headers and on this file (its flags), so a flag change rebuilds
    headers = (list(INC.glob("*.h")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) +
               [Path(__file__).resolve()])
    objs = []
    for src, extra in CUDA_SOURCES.items():
        s = CSRC / src
        o = OBJ / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            flags = NVCC_FLAGS + extra + (["-Xptxas", "-v"] if ptxas_info else [])
            _run([nvcc, *flags, "-c", str(s), "-o", str(o)], verbose or ptxas_info)
    for src in C_SOURCES:
        s = CSRC / src
        o = OBJ / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            _run([gcc, *C_FLAGS, "-c", str(s), "-o", str(o)], verbose)
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lm"], verbose)
    main_c = CSRC / "main.c"
    if main_c.exists() and _stale(CLI, [main_c, LIB] + headers):
        _run([gcc, *C_FLAGS, "-o", str(CLI), str(main_c), f"-L{PKG}", "-ldsmc_b200",
              "-Wl,-rpath,$ORIGIN/..", "-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
