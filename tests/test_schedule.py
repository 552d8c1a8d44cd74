"""The batched-solve schedule and its autotuner (gs_screen_tune, gs_grid_schedule_get / _set), on a B200 through the
C ABI: the tuner times its candidates on a sample screen and keeps the fastest; a screen's statuses, iterations and
violations do not depend on the schedule and its converged states agree to within 1e-10 (the same pieces of work whichever
kernel runs them; a level kernel and a persistent walk may add a dot product's terms in another order, which only an
outage that never converges carries far), and under the tuned schedule they still equal the oracle's."""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grid2000():
    m = synthetic.config_grid(1, 0)
    idx = synthetic.outage_set(m, None, 0)
    return m, idx


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_tuned_schedule_keeps_the_screen_equal_to_the_oracle(grid2000, precision):
    m, idx = grid2000
    opt = PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True, warm_start_from_base=True,
                           precision=precision)
    solver = SparseNewtonRaphsonPowerFlow(precision)
    g = solver.grid_for(m, opt)
    assert g.schedule() == {"factor_cut": 2, "solve_cut": 2, "tail_max": 296, "subtree_cut": -1}
    t = ContingencyAnalysis.tune_screen(m, idx[:600], solver, opt)
    assert t["factor_cut"] in (1, 2, 4) and t["solve_cut"] in (1, 2, 4) and t["tail_max"] in (74, 148, 296)
    assert t["candidates"] >= 8 and t["subtree_cut"] >= -1
    assert 0 < t["tuned_ms"] <= t["default_ms"]
    assert g.schedule() == {k: t[k] for k in ("factor_cut", "solve_cut", "tail_max", "subtree_cut")}
    got = ContingencyAnalysis.screen_raw(m, idx, solver, opt, keep_states=True)
    ref = oracle.screen(m, idx, PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True,
                                                 warm_start_from_base=True).to_c(), keep_states=True)
    assert np.array_equal(got["status"], ref["status"])
    assert np.array_equal(got["iterations"], ref["iterations"])
    conv = ref["status"] == _abi.PF_CONVERGED
    assert np.max(np.abs(got["vm"][conv] - ref["vm"][conv])) <= 1e-8
    assert np.max(np.abs(np.radians(got["va_deg"][conv] - ref["va_deg"][conv]))) <= 1e-8
    assert np.array_equal(got["viol_ptr"], ref["viol_ptr"]) and np.array_equal(got["viol_element"], ref["viol_element"])


def test_results_do_not_depend_on_the_schedule(grid2000):
    m, idx = grid2000
    opt = PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True, warm_start_from_base=True,
                           precision="mixed")
    solver = SparseNewtonRaphsonPowerFlow("mixed")
    g = solver.grid_for(m, opt)
    runs = []
    for sched in ({"factor_cut": 2, "solve_cut": 2, "tail_max": 296, "subtree_cut": -1},
                  {"factor_cut": 1, "solve_cut": 4, "tail_max": 74, "subtree_cut": 4},
                  {"factor_cut": 4, "solve_cut": 1, "tail_max": 148, "subtree_cut": 12},
                  {"factor_cut": 2, "solve_cut": 2, "tail_max": 296, "subtree_cut": 30}):
        g.set_schedule(**sched)
        got = g.schedule()
        assert {k: got[k] for k in ("factor_cut", "solve_cut", "tail_max")} == \
            {k: sched[k] for k in ("factor_cut", "solve_cut", "tail_max")}
        assert -1 <= got["subtree_cut"] <= sched["subtree_cut"]  # kept below the persistent walk
        runs.append(ContingencyAnalysis.screen_raw(m, idx, solver, opt, keep_states=True))
    conv = runs[0]["status"] == _abi.PF_CONVERGED
    for r in runs[1:]:
        assert np.array_equal(r["status"], runs[0]["status"])
        assert np.array_equal(r["iterations"], runs[0]["iterations"])
        assert np.max(np.abs(r["vm"][conv] - runs[0]["vm"][conv])) <= 1e-10
        assert np.max(np.abs(np.radians(r["va_deg"][conv] - runs[0]["va_deg"][conv]))) <= 1e-10
        assert np.array_equal(r["viol_ptr"], runs[0]["viol_ptr"])
        assert np.array_equal(r["viol_element"], runs[0]["viol_element"])
    with pytest.raises(RuntimeError):
        g.set_schedule(factor_cut=0)
