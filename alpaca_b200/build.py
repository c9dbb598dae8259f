"""Builds the CUDA library libalpaca_b200.so in-tree for sm_100a (nvcc).

Every source is compiled to its own object under alpaca_b200/_build/, in
parallel, and only when it (or a header) changed since its object was built;
the objects are then linked into the shared libraries.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libalpaca_b200.so")
PROBE_LIB = os.path.join(HERE, "libalpaca_b200_probe.so")
# Same sources without FMA contraction: every multiply and add is rounded on
# its own, as in the reference's x86-64 build. Tests use it to show that the
# CUDA arithmetic follows the reference's operation order bit for bit.
STRICT_LIB = os.path.join(HERE, "libalpaca_b200_strict.so")
SOURCES = ["kernels.cu", "capi.cu", "server.cu", "levels.cu", "static_scratch.cu", "ic_expr.cu",
           "elastic.cu",
           "tile_step.cu", "tile_step_fvchar.cu", "tile_step_fvprim.cu", "tile_step_fsroe.cu"]
PROBE_SOURCES = ["probe.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]
# only the alp_* C ABI is exported (exports.map)
LFLAGS = ["--shared", "-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map")]
VARIANTS = {"fast": (LIB, SOURCES, []),
            "strict": (STRICT_LIB, SOURCES, ["-fmad=false", "-DALP_STRICT"]),
            "probe": (PROBE_LIB, PROBE_SOURCES, [])}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps_mtime(path: str, seen=None) -> float:
    """Latest modification time of a source and the local headers it includes,
    followed recursively."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return 0.0
    seen.add(path)
    t = os.path.getmtime(path)
    with open(path) as f:
        for inc in _INCLUDE.findall(f.read()):
            t = max(t, _deps_mtime(os.path.join(os.path.dirname(path), inc), seen))
    return t


def _obj(variant: str, src: str) -> str:
    return os.path.join(OBJ, variant, src[:-3] + ".o")


def _stale(target: str, deps_mtime: float) -> bool:
    return not os.path.exists(target) or os.path.getmtime(target) < deps_mtime


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout[-6000:] + r.stderr[-6000:])


def stale() -> bool:
    for variant, (lib, sources, _) in VARIANTS.items():
        if not os.path.exists(lib):
            return True
        for s in sources:
            if _stale(lib, _deps_mtime(os.path.join(CSRC, s))):
                return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    jobs = []
    for variant, (lib, sources, extra) in VARIANTS.items():
        os.makedirs(os.path.join(OBJ, variant), exist_ok=True)
        for s in sources:
            o = _obj(variant, s)
            if force or _stale(o, _deps_mtime(os.path.join(CSRC, s))):
                jobs.append([nvcc()] + ARCH + CFLAGS + list(extra) +
                            ["-c", "-o", o, os.path.join(CSRC, s)])
    if jobs:
        # the largest translation units first
        jobs.sort(key=lambda c: -os.path.getsize(c[-1]))
        with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
            for f in [ex.submit(_run, j, verbose) for j in jobs]:
                f.result()
    for variant, (lib, sources, _) in VARIANTS.items():
        objs = [_obj(variant, s) for s in sources]
        if force or jobs or not os.path.exists(lib) or any(_stale(lib, os.path.getmtime(o)) for o in objs):
            _run([nvcc()] + ARCH + LFLAGS + ["-o", lib] + objs, verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
