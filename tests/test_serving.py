"""The request loop (gs_serve_*) on a B200, through the C ABI.

Results are held to the parity bar of the other GPU tests against the oracle (identical statuses, converged
voltages within 1e-8 pu and angles within 1e-8 rad), and a request's result must be the same whether it runs
alone or among hundreds of others on several grids: the same status and iteration count, and states equal
within SAME_TOL (a system's arithmetic does not depend on its slot or its neighbours, so in practice they are
bit-identical).
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import EngineError, PowerFlowOptions
from gridsim_b200.serving import LoadFlowServer, drain
from tests.conftest import golden_model

pytestmark = pytest.mark.gpu

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8
SAME_TOL = 1e-12


def _opts(precision="mixed"):
    return PowerFlowOptions(precision=precision, max_iterations=20, warm_start_from_base=True,
                            per_bus_voltage_limits=True)


@pytest.fixture(scope="module")
def population():
    case118, _ = golden_model("case118")
    grids = [synthetic.config_grid(0, 0), case118, synthetic.make_grid(600, 825, 72, seed=5)]
    outages = [synthetic.outage_set(grids[0], 40, 1), case118.in_service_branches()[:40],
               synthetic.outage_set(grids[2], 40, 2)]
    return grids, outages


def _start(grids, precision="mixed", slots=32):
    srv = LoadFlowServer(_opts(precision), slots_per_grid=slots)
    for m in grids:
        srv.add_grid(m)
    srv.start()
    return srv


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_requests_match_the_oracle(population, precision):
    grids, outages = population
    srv = _start(grids, precision)
    try:
        reqs = []
        for g, idx in enumerate(outages):
            reqs.append((g, -1, 1))
            reqs.extend((g, int(k), 1) for k in idx)
        tickets = srv.submit(reqs)  # more requests per grid than slots: the rest wait for free slots
        got = {r.ticket: r for r in drain(srv, len(reqs))}
        assert sorted(got) == sorted(int(t) for t in tickets)
        opt = _opts(precision).to_c()
        for g, (m, idx) in enumerate(zip(grids, outages)):
            base = oracle.solve(m, opt)
            ref = oracle.screen(m, idx, opt, keep_states=True)
            n = m.n_bus
            for j, (req, t) in enumerate(zip(reqs, tickets)):
                if req[0] != g:
                    continue
                r = got[int(t)]
                if req[1] < 0:
                    st, vm, va = base["status"], base["vm"], base["va_deg"]
                else:
                    k = int(np.nonzero(idx == req[1])[0][0])
                    st = ref["status"][k]
                    vm = np.asarray(ref["vm"]).reshape(len(idx), n)[k]
                    va = np.asarray(ref["va_deg"]).reshape(len(idx), n)[k]
                if st == _abi.PF_UNSOLVABLE_PART:
                    # the screen reports a provably unsolvable outage without solving it; a request is a solve
                    # (IPowerFlowSolver.Solve), which can only end unconverged there
                    assert r.status != _abi.PF_CONVERGED, (g, req)
                    continue
                assert r.status == st, (g, req)
                if st == _abi.PF_CONVERGED:
                    assert r.max_mismatch < 1e-8
                    assert np.max(np.abs(r.vm - vm)) <= VM_TOL, (g, req)
                    assert np.max(np.abs(np.radians(r.va_deg - va))) <= VA_TOL_RAD, (g, req)
        st = srv.stats()
        assert st["completed"] == st["submitted"] == len(reqs) and st["failed"] == 0
    finally:
        srv.close()


def test_result_is_the_same_alone_and_in_the_mix(population):
    grids, outages = population
    srv = _start(grids)
    try:
        probes = [(0, int(outages[0][3]), 1), (1, -1, 1), (2, int(outages[2][7]), 1), (1, int(outages[1][11]), 1)]
        alone = []
        for p in probes:  # each on its own, nothing else in flight
            t = srv.submit([p])
            (r,) = drain(srv, 1)
            assert r.ticket == int(t[0])
            alone.append(r)
        rng = np.random.default_rng(7)
        mix = []
        for _ in range(400):
            g = int(rng.integers(0, len(grids)))
            o = -1 if rng.random() < 0.5 else int(rng.choice(outages[g]))
            mix.append((g, o, 0))
        reqs = mix[:150] + probes[:2] + mix[150:300] + probes[2:] + mix[300:]
        tickets = srv.submit(reqs)
        got = {r.ticket: r for r in drain(srv, len(reqs))}
        pos = [150, 151, 302, 303]
        for a, p in zip(alone, pos):
            b = got[int(tickets[p])]
            assert (b.grid, b.outage) == (a.grid, a.outage)
            assert b.status == a.status and b.iterations == a.iterations
            assert b.max_mismatch == a.max_mismatch or abs(b.max_mismatch - a.max_mismatch) <= SAME_TOL
            assert np.max(np.abs(b.vm - a.vm)) <= SAME_TOL
            assert np.max(np.abs(b.va_deg - a.va_deg)) <= SAME_TOL
    finally:
        srv.close()


def test_many_more_requests_than_slots(population):
    grids, outages = population
    srv = _start(grids[:1], slots=32)
    try:
        reqs = [(0, int(outages[0][k % len(outages[0])])) for k in range(1000)]
        tickets = srv.submit(reqs)
        res = drain(srv, len(reqs))
        assert len({r.ticket for r in res}) == len(reqs) == len(set(int(t) for t in tickets))
        assert all(r.latency_ms >= r.queue_ms >= 0 for r in res)
        st = srv.stats()
        assert st["completed"] == 1000 and st["ticks"] > 0 and st["system_steps"] >= sum(r.iterations for r in res)
        srv.stop()
        with pytest.raises(EngineError):
            srv.submit([(0, -1)])
    finally:
        srv.close()


def test_slots_grow_with_queued_requests_within_the_memory_budget(population):
    """Admission by device memory: a grid starts with 32 slots and takes 32 more at a time while its requests queue
    and the loop's budget holds them; results equal the oracle's whatever width the batch has grown to. With a
    budget that holds only the first 32 slots, the grid stays at 32 and every request is still answered."""
    import torch
    grids, outages = population
    m, idx = grids[0], outages[0]
    opt = _opts().to_c()
    ref = oracle.screen(m, idx, opt, keep_states=True)
    reqs = [(0, int(idx[k % len(idx)]), 1) for k in range(600)]
    srv = LoadFlowServer(_opts(), slots_per_grid=128)
    try:
        srv.add_grid(m)
        first = srv.stats()
        assert first["slots_total"] == 32
        srv.start()
        tickets = srv.submit(reqs)
        got = {r.ticket: r for r in drain(srv, len(reqs))}
        st = srv.stats()
        assert st["slots_total"] > 32 and st["slot_bytes"] > first["slot_bytes"]
        n = m.n_bus
        for req, t in zip(reqs, tickets):
            k = int(np.nonzero(idx == req[1])[0][0])
            r = got[int(t)]
            assert r.status == ref["status"][k]
            if r.status == _abi.PF_CONVERGED:
                assert np.max(np.abs(r.vm - np.asarray(ref["vm"]).reshape(len(idx), n)[k])) <= VM_TOL
                assert np.max(np.abs(np.radians(r.va_deg - np.asarray(ref["va_deg"]).reshape(len(idx), n)[k]))) <= VA_TOL_RAD
    finally:
        srv.close()
    # a budget for the first 32 slots only (their bytes with a 20 % margin, as a share of the free memory now)
    free, _ = torch.cuda.mem_get_info()
    srv = LoadFlowServer(_opts(), slots_per_grid=128, hbm_fraction=1.2 * first["slot_bytes"] / free)
    try:
        srv.add_grid(m)
        srv.start()
        srv.submit(reqs)
        res = drain(srv, len(reqs))
        assert len(res) == len(reqs)
        assert srv.stats()["slots_total"] == 32
    finally:
        srv.close()


def test_bad_requests_are_refused(population):
    grids, _ = population
    srv = LoadFlowServer(_opts(), slots_per_grid=32)
    try:
        g = srv.add_grid(grids[0])
        with pytest.raises(EngineError):
            srv.submit([(g, -1)])  # not started
        srv.start()
        with pytest.raises(EngineError):
            srv.submit([(g + 1, -1)])  # unknown grid
        with pytest.raises(EngineError):
            srv.submit([(g, grids[0].n_branch)])  # no such branch
        with pytest.raises(EngineError):
            LoadFlowServer(_opts(), slots_per_grid=48)  # not a multiple of 32
    finally:
        srv.close()


def test_requests_with_q_limits_and_the_retry_are_answered_in_batches():
    """The reference's rpc solve options (100 iterations, Q limits on, the DC retry on: RpcCommand.cs:675-676): the
    loop answers them through batch solves, held to the oracle like the slot-stepped requests."""
    from gridsim_b200.engine import study_options
    from tests.conftest import assert_states_close

    m, _ = golden_model("case118")
    opt = study_options()
    idx = m.in_service_branches()[:30]
    srv = LoadFlowServer(opt)
    try:
        g = srv.add_grid(m)
        srv.start()
        reqs = [(g, -1, 1)] * 3 + [(g, int(k), 1) for k in idx]
        tickets = srv.submit(reqs)
        got = {r.ticket: r for r in drain(srv, len(reqs))}
        base = oracle.solve(m, opt.to_c())
        ref = oracle.screen(m, idx, opt.to_c(), keep_states=True)
        for j, (req, t) in enumerate(zip(reqs, tickets)):
            r = got[int(t)]
            if req[1] < 0:
                assert r.status == base["status"] == _abi.PF_CONVERGED
                assert np.max(np.abs(r.vm - base["vm"])) <= VM_TOL
                assert np.max(np.abs(np.radians(r.va_deg - base["va_deg"]))) <= VA_TOL_RAD
                continue
            k = j - 3
            if ref["status"][k] == _abi.PF_UNSOLVABLE_PART:
                assert r.status != _abi.PF_CONVERGED
                continue
            assert r.status == ref["status"][k], req
            if r.status == _abi.PF_CONVERGED:
                assert_states_close(m, [req[1]], r.vm, r.va_deg, ref["vm"][k], ref["va_deg"][k], VM_TOL, VA_TOL_RAD)
        st = srv.stats()
        assert st["completed"] == st["submitted"] == len(reqs) and st["failed"] == 0
    finally:
        srv.close()


def test_warm_starts_with_q_limits_are_refused():
    from gridsim_b200.engine import study_options

    opt = study_options()
    opt.warm_start_from_base = True
    with pytest.raises(EngineError):
        LoadFlowServer(opt)
