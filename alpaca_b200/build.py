"""Builds the CUDA library libalpaca_b200.so in-tree for sm_100a (nvcc)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libalpaca_b200.so")
PROBE_LIB = os.path.join(HERE, "libalpaca_b200_probe.so")
# Same sources without FMA contraction: every multiply and add is rounded on
# its own, as in the reference's x86-64 build. Tests use it to show that the
# CUDA arithmetic follows the reference's operation order bit for bit.
STRICT_LIB = os.path.join(HERE, "libalpaca_b200_strict.so")
SOURCES = ["kernels.cu", "capi.cu", "server.cu", "levels.cu", "static_scratch.cu", "ic_expr.cu"]
PROBE_SOURCES = ["probe.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# only the alp_* C ABI is exported (exports.map)
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--shared",
         "-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map")]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(os.path.dirname(HERE), "include", "alpaca_b200.h")
    return os.path.getmtime(hdr) > t


def _nvcc(out: str, sources: list[str], verbose: bool, extra=()) -> None:
    cmd = [nvcc()] + ARCH + FLAGS + list(extra) + ["-o", out] + [os.path.join(CSRC, s) for s in sources]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout[-6000:] + r.stderr[-6000:])


def build(force: bool = False, verbose: bool = False) -> str:
    if force or stale() or not os.path.exists(PROBE_LIB) or not os.path.exists(STRICT_LIB):
        _nvcc(LIB, SOURCES, verbose)
        _nvcc(STRICT_LIB, SOURCES, verbose, ["-fmad=false", "-DALP_STRICT"])
        _nvcc(PROBE_LIB, PROBE_SOURCES, verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
