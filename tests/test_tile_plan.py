"""CPU replay of the fused tile kernel's plan (tile_plan.cuh): the TMA boxes,
the ring of x-planes and the halo / U0 buffers, the warp-task stream and its
bookkeeping, for every combination of neighbour, zero-gradient and symmetry
faces. Every face is computed exactly once from the stencil the pool holds,
no buffer is reused while a task still reads it, and every wait is satisfied
in stream order (no cycle). The replay links the plan header itself
(tests/tile_plan_emu.cpp)."""
import itertools
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("tile") / "tile_plan_emu")
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wno-unknown-pragmas", "-o", exe,
                    os.path.join(HERE, "tile_plan_emu.cpp")], check=True)
    return exe


KINDS = list(itertools.product((0, 1, 2), repeat=2))


@pytest.mark.parametrize("x", KINDS)
@pytest.mark.parametrize("yz", [(0, 0, 0, 0), (1, 2, 2, 1), (2, 0, 1, 1), (0, 2, 0, 1)])
def test_tile_plan_replay(emu, x, yz):
    r = subprocess.run([emu] + [str(k) for k in x + yz], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split() == ["ok", str(3 * 17 * 256), "4096"]
