"""Device-evaluated initial conditions and the serving request loop (alp_serve)."""
import numpy as np
import pytest

import oracle
from alpaca_b200 import api, cases, serving
from alpaca_b200 import native as N
from helpers import l1_rel

pytestmark = pytest.mark.gpu


def host_ic(req: serving.Request) -> np.ndarray:
    """The request's initial condition evaluated with numpy (same formulas)."""
    dim = req.dim
    g = cases.BlockGrid(dim, req.nblocks[:dim], tuple(bool(p) for p in req.periodic[:dim]),
                        req.cell_size)
    x = g.cell_centres()
    q = req.params
    if req.ic_type == N.IC_QUADRANTS:
        quad = (x[0] >= q[0]).astype(int) + 2 * (x[1] >= q[1]).astype(int)
        s = np.array(q[2:18]).reshape(4, 4)
        rho, u, v, p = (s[quad, i] for i in range(4))
        vel = [u, v]
    else:
        r2 = sum((x[d] - q[d]) ** 2 for d in range(dim))
        inside = r2 < q[3] * q[3]
        rho = np.where(inside, q[4], q[6])
        p = np.where(inside, q[5], q[7])
        vel = [np.zeros_like(rho) for _ in range(dim)]
    glob = cases.primes_to_conservatives(dim, rho, p, vel, req.gamma, req.B)
    return g.scatter(glob), g


@pytest.mark.parametrize("kind", ["quadrants", "blast_gas", "blast_water"])
def test_device_initial_condition_matches_host(cuda, kind):
    rng = np.random.default_rng(4)
    if kind == "quadrants":
        req = serving.quadrant_request(rng, 6, 5)
    else:
        req = serving.blast_request(rng, 8, 5, water=kind == "blast_water")
    u_host, g = host_ic(req)
    eng = api.Engine(req.dim, "fvchar", capacity_blocks=g.nb, max_cases=1)
    cid = eng.add_case_ic(req.ic_type, req.params, req.nblocks, req.cell_size,
                          N.Material.make(req.gamma, req.B), max_steps=5)
    u_dev = eng.get(cid)[0]
    I = cases.interior(req.dim)
    np.testing.assert_allclose(u_dev[I], u_host[I], rtol=1e-15, atol=0)
    # the device-generated case steps exactly like the oracle on the same state
    eng.run_to_end(chunk=5)
    got, t, steps = eng.get(cid)
    eng.close()
    ref = oracle.Restatement(req.dim, "fvchar").run(u_dev, g.nbr, req.gamma, req.B, False,
                                                    req.cell_size, 0.6, 1e300, max_steps=5)[0]
    assert steps == 5
    for f in range(req.dim + 2):
        assert l1_rel(got[I][:, f], ref[I][:, f]) <= 1e-12


def small_stream(seed=2):
    """Five small cases that all arrive at once (so the batched run overlaps them)."""
    rng = np.random.default_rng(seed)
    reqs = [serving.quadrant_request(rng, 4, 30), serving.blast_request(rng, 8, 20, water=False),
            serving.blast_request(rng, 27, 12, water=True), serving.quadrant_request(rng, 12, 25),
            serving.blast_request(rng, 8, 16, water=False)]
    for r in reqs:
        r.arrival_s = 0.0
    return reqs


def test_serving_mix_equals_alone(cuda):
    """Continuous batching gives each case the same bits it gets alone."""
    reqs = small_stream()
    budget = 2 << 30
    mix, _, states_mix = api.serve(reqs, budget, keep_results=True)
    alone, _, states_alone = api.serve(reqs, budget, one_at_a_time=True, keep_results=True)
    for i, r in enumerate(reqs):
        assert mix[i]["status"] == 0 and alone[i]["status"] == 0
        assert mix[i]["steps"] == alone[i]["steps"] == r.max_steps
        assert np.array_equal(states_mix[i][cases.interior(r.dim)],
                              states_alone[i][cases.interior(r.dim)]), i
    # one at a time: no two cases resident together
    spans = sorted((x["admitted_s"], x["finished_s"]) for x in alone)
    for (a0, f0), (a1, _) in zip(spans, spans[1:]):
        assert a1 >= f0
    # batched: cases overlap on the device
    mspans = sorted((x["admitted_s"], x["finished_s"]) for x in mix)
    assert any(a1 < f0 for (a0, f0), (a1, _) in zip(mspans, mspans[1:]))


def test_serving_program_requests(cuda):
    """Requests whose initial condition is an expression program: batched with
    fixed-form requests they get the bits they get alone and the bits of the
    engine's own expression case."""
    prog2 = api.IcProgram("""if ((x < 0.5) & (y < 0.5)) { density := 1; pressure := 1; }
        else { density := 0.125 + 0.1 * sin(2 * pi * y); pressure := 0.1; velocityX := 0.2; }""")
    prog3 = api.IcProgram("""var r := sqrt((x - 0.25)^2 + (y - 0.25)^2 + (z - 0.25)^2);
        density := r < 0.1 ? 2.0 : 1.0; pressure := r < 0.1 ? 10.0 : 1.0;""")
    reqs = [
        serving.Request(2, (4, 4, 1), 1.0 / 64, 1.4, 0.0, N.IC_PROGRAM, [], 20, program=prog2),
        serving.Request(3, (2, 2, 2), 1.0 / 64, 1.4, 0.0, N.IC_PROGRAM, [], 12, arrival_s=0.01,
                        program=prog3, units=(1.0, 1.0, 2.0)),
    ] + small_stream()[:3]
    budget = 2 << 30
    mix, _, states_mix = api.serve(reqs, budget, keep_results=True)
    alone, _, states_alone = api.serve(reqs, budget, one_at_a_time=True, keep_results=True)
    for i, r in enumerate(reqs):
        assert mix[i]["status"] == 0 and alone[i]["status"] == 0
        I = cases.interior(r.dim)
        assert np.array_equal(states_mix[i][I], states_alone[i][I]), i
    for i, (prog, units) in enumerate(((prog2, None), (prog3, N.Units(1.0, 1.0, 2.0)))):
        r = reqs[i]
        eng = api.Engine(r.dim, "fvchar", capacity_blocks=r.blocks, max_cases=1)
        cid = eng.add_case_expr(prog, r.nblocks, r.cell_size, N.Material.make(1.4),
                                max_steps=r.max_steps, units=units)
        eng.step(r.max_steps)
        u = eng.get(cid)[0]
        eng.close()
        I = cases.interior(r.dim)
        assert np.array_equal(u[I], states_mix[i][I]), i
    prog2.close()
    prog3.close()


def test_shortest_first_finishes_short_cases_first_with_the_same_bits(cuda):
    """Shortest remaining work first: a small case that arrives with large ones
    finishes before them, and every case keeps the bits it gets alone."""
    rng = np.random.default_rng(12)
    big = [serving.blast_request(rng, 27, 60, water=False) for _ in range(2)]
    small = serving.quadrant_request(rng, 4, 20)
    reqs = big + [small]
    for r in reqs:
        r.arrival_s = 0.0
    budget = 2 << 30
    # step set of one big case: the small case and one big case step, the
    # other big case waits
    res, _, st = api.serve(reqs, budget, keep_results=True, shortest_first=True,
                           step_set_cells=27 * 4096.0, steps_per_poll=4)
    alone, _, st_alone = api.serve(reqs, budget, one_at_a_time=True, keep_results=True)
    for i, r in enumerate(reqs):
        assert res[i]["status"] == 0 and res[i]["steps"] == r.max_steps
        assert np.array_equal(st[i][cases.interior(r.dim)], st_alone[i][cases.interior(r.dim)]), i
    assert res[2]["finished_s"] < min(res[0]["finished_s"], res[1]["finished_s"])
    # the held big case finishes after the other one (it waited)
    assert res[1]["finished_s"] > res[0]["finished_s"]


def test_serving_budget_bounds_admission(cuda):
    """With a budget for one 8-block 3D case, requests are admitted one after
    the other and all complete."""
    rng = np.random.default_rng(9)
    reqs = [serving.blast_request(rng, 8, 6, water=False) for _ in range(3)]
    per_block = N.lib().alp_engine_bytes(3, 1, 0)
    res, makespan, _ = api.serve(reqs, 9 * per_block)
    assert all(r["status"] == 0 and r["steps"] == 6 for r in res)
    spans = sorted((x["admitted_s"], x["finished_s"]) for x in res)
    for (a0, f0), (a1, _) in zip(spans, spans[1:]):
        assert a1 >= f0
    assert makespan >= spans[-1][1]


def test_serving_fp32_flux_within_target(cuda):
    """The FP32-flux form serves the same cases within 1e-5 relative L1 density."""
    reqs = small_stream(5)
    budget = 2 << 30
    r64, _, s64 = api.serve(reqs, budget, keep_results=True)
    r32, _, s32 = api.serve(reqs, budget, precision=N.FP32_FLUX, keep_results=True)
    for i, r in enumerate(reqs):
        I = cases.interior(r.dim)
        err = l1_rel(s32[i][I][:, 0], s64[i][I][:, 0])
        assert r32[i]["steps"] == r64[i]["steps"] and err <= 1e-5, (i, err)


def test_serving_request_too_large_is_reported(cuda):
    rng = np.random.default_rng(1)
    big = serving.blast_request(rng, 64, 3, water=False)
    small = serving.blast_request(rng, 1, 3, water=False)
    per_block = N.lib().alp_engine_bytes(3, 1, 0)
    res, _, _ = api.serve([big, small], 8 * per_block)
    assert res[0]["status"] == N.ALP_ERR_CAPACITY
    assert res[1]["status"] == 0 and res[1]["steps"] == 3


def test_abort_file_stops_serving_cleanly(cuda, tmp_path):
    """The reference stops a run when its ABORTFILE appears; alp_serve checks
    its abort file after every poll. Present from the start, one case (one at
    a time) has taken one poll of steps when the loop stops: that case comes
    back with its state and steps, the others with none, all ALP_ABORTED."""
    stop = tmp_path / "ABORTFILE"
    stop.write_text("")
    reqs = small_stream()
    res, _, states = api.serve(reqs, 2 << 30, one_at_a_time=True, steps_per_poll=4,
                               keep_results=True, abort_file=str(stop))
    assert all(x["status"] == N.ALP_ABORTED for x in res)
    ran = [i for i, x in enumerate(res) if x["steps"] > 0]
    assert len(ran) == 1 and res[ran[0]]["steps"] == 4 and res[ran[0]]["t"] > 0.0
    I = cases.interior(reqs[ran[0]].dim)
    assert np.isfinite(states[ran[0]][I]).all() and (states[ran[0]][I][:, 0] > 0).all()
    assert all(x["steps"] == 0 and x["t"] == 0.0 for i, x in enumerate(res) if i != ran[0])
    # without the file the same stream runs to the end
    stop.unlink()
    done, _, _ = api.serve(reqs, 2 << 30, one_at_a_time=True, steps_per_poll=4,
                           abort_file=str(stop))
    assert all(x["status"] == 0 and x["steps"] == r.max_steps for x, r in zip(done, reqs))


def test_abort_file_while_waiting_for_arrivals(cuda, tmp_path):
    """With nothing resident the loop still checks its abort file: every
    request arrives seconds after the start and the file exists from the
    start, so alp_serve returns ALP_ABORTED at once, nothing admitted and no
    step taken."""
    import time
    stop = tmp_path / "ABORTFILE"
    stop.write_text("")
    reqs = small_stream()
    for r in reqs:
        r.arrival_s = 5.0
    t0 = time.perf_counter()
    res, mk, _ = api.serve(reqs, 2 << 30, steps_per_poll=4, abort_file=str(stop))
    assert time.perf_counter() - t0 < 3.0 and mk < 3.0
    assert all(x["status"] == N.ALP_ABORTED and x["steps"] == 0 and x["t"] == 0.0 and
               x["admitted_s"] < 0.0 for x in res)
