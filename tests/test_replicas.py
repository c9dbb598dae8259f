"""The N>1 path of bench.py on CPU ranks (gloo, world size 2): every rank
advances its own copy of the case (replicas, no data-path collective), the
timing is the max over ranks and the value aggregates all ranks' cells."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import types

    import bench
    import oracle
    from alpaca_b200 import cases
    args = types.SimpleNamespace(impl="reference")  # gloo backend
    ws_, rank_, _ = bench.dist_setup(args)
    assert (ws_, rank_) == (ws, rank)
    case = cases.fourier_shock(1, dim=3, seed=40 + rank, steps=2)
    bench.barrier(ws_)
    import time
    t0 = time.perf_counter()
    u = oracle.Restatement(3).run(case.u, case.grid.nbr, 1.4, 0.0, False, case.grid.cell_size,
                                  0.6, 1e300, max_steps=2)[0]
    local = (time.perf_counter() - t0) + 0.05 * rank  # ranks differ in time
    tmax = bench.max_over_ranks(local, ws_)
    bench.barrier(ws_)
    out[rank] = (local, tmax, float(np.abs(u).sum()))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_cpu_ranks_max_time_and_independent_replicas():
    ws = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_rank, args=(ws, port, out), nprocs=ws, join=True, start_method="spawn")
    local = [out[r][0] for r in range(ws)]
    for r in range(ws):
        assert out[r][1] == pytest.approx(max(local))
    # independent seeds -> independent states (no exchange between replicas)
    assert out[0][2] != out[1][2]
