"""Multi-level halos against the reference's own glue (no GPU).

oracle/_ref/libalpglue_d3.so runs ALPACA's TopologyManager, Tree, Averager
(AverageMaterial, multiresolution/averager.cpp:62) and InternalHaloManager
(same-level copies and the jump halos of UpdateMaterialJumpNoMpi,
communication/internal_halo_manager.cpp:230-290) on one rank against the
single-rank MPI stand-in oracle/mpi_shim/mpi.h. The restatement's level halos
(oracle_level_halos: what a stage of the level step, and the CUDA level path
that is bit-exact with it, reads beyond each leaf's faces) must equal the
reference's bit for bit on every face towards another leaf: same level,
finer (averaged) and coarser (predicted) neighbours.
"""
import numpy as np
import pytest

import oracle
from alpaca_b200 import cases

pytestmark = pytest.mark.skipif(not oracle.Glue.available(),
                                reason="reference glue not built (reference sources absent)")

IC, HS = 16, 4


def centred_hierarchy():
    """4^3 level-0 nodes; the central 2^3 refined, and inside them two
    level-1 nodes refined again (2:1 balance enforced by the tree builder),
    so that every jump lies at least one level-0 node away from the domain
    faces. Smooth seeded fields in every leaf."""
    def refine(l, lo, hi):
        if l == 0:
            return all(1.0 <= lo[d] < 3.0 for d in range(3))
        return any(np.allclose(lo, c) for c in ((1.5, 1.5, 1.5), (2.0, 1.5, 1.5)))
    case = cases.spherical_shock_levels(n0=4, dim=3, lmax=2, refine=refine)
    rng = np.random.default_rng(17)
    k = rng.uniform(0.5, 2.0, size=(5, 3))
    ph = rng.uniform(0.0, 2 * np.pi, size=5)
    I = cases.interior(3)
    u = np.zeros_like(case.u)
    for b in range(case.nleaf):
        x = case.cell_centres(b)
        f = [np.sin(2 * np.pi * (k[i, 0] * x[0] + k[i, 1] * x[1] + k[i, 2] * x[2]) + ph[i])
             for i in range(5)]
        rho, p = 1.0 + 0.2 * f[0], 1.0 + 0.1 * f[1]
        vel = [0.3 * f[2], 0.2 * f[3], 0.1 * f[4]]
        u[(b, slice(None)) + I[1:]] = cases.primes_to_conservatives(3, rho, p, vel, 1.4)
    return case, u


def face_halo(d, s):
    """Index of the face halo of direction d, side s (-1 low, +1 high):
    HS layers beyond the face over the interior extent."""
    sl = [slice(HS, HS + IC)] * 3
    sl[d] = slice(HS + IC, HS + IC + HS) if s > 0 else slice(0, HS)
    return (slice(None),) + tuple(sl)


def test_level_halos_equal_reference_glue():
    case, u = centred_hierarchy()
    assert case.leaves_per_level()[2] > 0
    ours = oracle.Restatement(3).level_halos(u, case.level, case.coord, case.n0)
    ref = oracle.Glue().level_halos(u, case.level, case.coord, case.n0)
    # the neighbour of every face at the leaf's level, to classify it
    where = {(int(case.level[b]), tuple(int(c) for c in case.coord[b])): b
             for b in range(case.nleaf)}
    kinds = {"same": 0, "finer": 0, "coarser": 0}
    for b in range(case.nleaf):
        l, c = int(case.level[b]), case.coord[b]
        for d in range(3):
            for s in (-1, 1):
                n = list(int(x) for x in c)
                n[d] += s
                if n[d] < 0 or n[d] >= 4 << l:
                    continue  # domain face: filled by the external boundary, not compared
                if (l, tuple(n)) in where:
                    kind = "same"
                elif any((l + 1, tuple(2 * n[e] + ((o >> e) & 1) for e in range(3))) in where
                         for o in range(8)):
                    kind = "finer"
                else:
                    kind = "coarser"
                kinds[kind] += 1
                h = face_halo(d, s)
                a, r = ours[b][h], ref[b][h]
                assert np.array_equal(a, r), (b, l, tuple(c), d, s, kind,
                                              float(np.abs(a - r).max()))
    assert all(v > 0 for v in kinds.values()), kinds
