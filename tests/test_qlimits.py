"""Q-limit enforcement (PV -> PQ switching passes, reverts of broken pins) on a B200, through the C ABI, against the
oracle's restatement of SparseNewtonRaphsonPowerFlow's Q-limit loop (NewtonShell.ApplyQLimits / RevertBrokenPins).

Parity bar as the other GPU tests: identical statuses and convergence flags, converged voltages within 1e-8 pu and
angles within 1e-8 rad, identical violation lists; plus the reference's own N-1 counts under StudyOptions
(ContingencyCorrectnessTests.cs:143-154 for case118, :209-237 for case14).
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow
from tests.conftest import golden_model

pytestmark = pytest.mark.gpu

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8


def _counts(status, viol_ptr):
    conv = status == _abi.PF_CONVERGED
    nv = np.diff(viol_ptr)
    return int(np.sum(conv & (nv == 0))), int(np.sum(conv & (nv > 0))), int(np.sum(~conv))


def _compare(gpu, ref):
    assert np.array_equal(gpu["status"], ref["status"]), "statuses differ"
    conv = ref["status"] == 0
    if conv.any():
        assert np.max(np.abs(gpu["vm"][conv] - ref["vm"][conv])) <= VM_TOL
        assert np.max(np.abs(np.radians(gpu["va_deg"][conv] - ref["va_deg"][conv]))) <= VA_TOL_RAD
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(gpu["viol_kind"], ref["viol_kind"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])


@pytest.mark.parametrize("name", ["case9", "case14", "case57", "case118", "case300"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_single_solve_with_q_limits_matches_oracle(name, precision):
    m, pub = golden_model(name)
    opt = PowerFlowOptions(precision=precision, enforce_q_limits=True)
    r = SparseNewtonRaphsonPowerFlow(precision).solve(m, opt)
    ref = oracle.solve(m, opt.to_c())
    assert r.status == ref["status"] == _abi.PF_CONVERGED
    assert r.iterations == ref["iterations"]
    assert np.max(np.abs(r.vm - ref["vm"])) <= VM_TOL
    assert np.max(np.abs(np.radians(r.va_deg - ref["va_deg"]))) <= VA_TOL_RAD
    slack = int(np.nonzero(m.bus_type == 3)[0][0])
    va = r.va_deg - r.va_deg[slack] + pub["va_deg"][slack]
    assert np.max(np.abs(r.vm - pub["vm"])) <= pub["vm_tol"]
    assert np.max(np.abs(va - pub["va_deg"])) <= pub["va_tol_deg"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_case118_n1_under_study_options(precision):
    m, _ = golden_model("case118")
    opt = PowerFlowOptions(max_iterations=100, enforce_q_limits=True, precision=precision)
    idx = m.in_service_branches()
    gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), opt, keep_states=True)
    ref = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    _compare(gpu, ref)
    assert _counts(gpu["status"], gpu["viol_ptr"]) == (164, 13, 9)


def test_case14_raw_counts_under_study_options():
    m, _ = golden_model("case14")
    opt = PowerFlowOptions(max_iterations=100, enforce_q_limits=True)
    idx = m.in_service_branches()
    gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow("fp64"), opt, keep_states=True)
    assert _counts(gpu["status"], gpu["viol_ptr"]) == (0, 19, 1)


@pytest.fixture(scope="module")
def tight_grid():
    """The 120-bus synthetic grid with reactive limits around each unit's base-case output, so that the outages
    push units onto their limits (and some back)."""
    m = synthetic.config_grid(0, 0)
    base = oracle.solve(m)
    qgen = base["q_inj_mvar"] + m.qd
    mt = m.copy()
    for k in range(m.n_gen):
        i = int(m.gen_bus[k])
        share = 1.0 / max(1, int(np.sum(m.gen_bus == i)))
        q = qgen[i] * share
        mt.qmax[k] = q + abs(q) * 0.05 + 0.5
        mt.qmin[k] = q - abs(q) * 0.05 - 0.5
    return mt


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tight_limits_n1_matches_oracle(tight_grid, precision):
    m = tight_grid
    opt = PowerFlowOptions(max_iterations=30, enforce_q_limits=True, warm_start_from_base=True,
                           per_bus_voltage_limits=True, precision=precision)
    idx = synthetic.outage_set(m, None, 0)
    gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), opt, keep_states=True)
    ref = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    _compare(gpu, ref)
    assert np.array_equal(gpu["iterations"], ref["iterations"])
    # the limits bind: without enforcement the states differ
    free = oracle.screen(m, idx, PowerFlowOptions(max_iterations=30, warm_start_from_base=True,
                                                  per_bus_voltage_limits=True).to_c(), keep_states=True)
    both = (free["status"] == 0) & (ref["status"] == 0)
    assert np.max(np.abs(free["vm"][both] - ref["vm"][both])) > 1e-4


def test_multi_grid_batch_takes_q_limits_through_batch_solves():
    """The uneven multi-grid batch runs Q-limit cases as each grid's batch solve: the same results bit for bit."""
    from gridsim_b200.engine import UnevenBatch
    m = synthetic.config_grid(0, 0)
    opt = PowerFlowOptions(enforce_q_limits=True)
    b = UnevenBatch([m])
    try:
        r = b.solve([2], options=opt, keep_states=True)
    finally:
        b.close()
    ref = SparseNewtonRaphsonPowerFlow().solve_batch(m, outage=np.array([-1, -1], np.int32), options=opt,
                                                     keep_states=True)
    assert np.array_equal(r["status"][0], ref["status"]) and (ref["status"] == 0).all()
    assert np.array_equal(r["vm"][0], ref["vm"]) and np.array_equal(r["va_deg"][0], ref["va_deg"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("extra", [{"revert_q_limits": True}, {"max_q_limit_passes": 1}, {"max_q_limit_passes": 3}])
def test_revert_and_pass_cap_options_match_the_oracle(tight_grid, precision, extra):
    """RevertQLimits (a pinned bus may go back to PV in the pass that switches others, PowerFlowOptions.cs:103-110) and
    MaxQLimitPasses (:100-101) on the tight-limits grid: both change the screen (checked on the oracle) and the device
    follows the oracle."""
    m = tight_grid
    opt = PowerFlowOptions(max_iterations=30, enforce_q_limits=True, warm_start_from_base=True,
                           per_bus_voltage_limits=True, precision=precision, **extra)
    idx = synthetic.outage_set(m, None, 0)
    gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), opt, keep_states=True)
    ref = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    _compare(gpu, ref)
    assert np.array_equal(gpu["iterations"], ref["iterations"])
    plain = oracle.screen(m, idx, PowerFlowOptions(max_iterations=30, enforce_q_limits=True, warm_start_from_base=True,
                                                   per_bus_voltage_limits=True).to_c())
    assert not np.array_equal(plain["iterations"], ref["iterations"])
