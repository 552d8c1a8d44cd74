"""The DC-angle retry (NewtonShell.SolveWithRetry / TrySeedDcAngles / Stalled): a solve whose Newton run stalls is
solved again from DC power-flow angles and kept when it converges with every branch angle within 90 degrees.

CPU: the oracle's restatement, from start angles scrambled by up to +-120 degrees: without the retry the solve stalls
at the iteration cap; with it the solve converges to the same root as from the case's own start (case118: the
published voltages, IeeeCasesTests.cs:16-24). GPU: the engine against the oracle on the same inputs (statuses,
iterations, converged voltages within 1e-8 pu and angles within 1e-8 rad, violation lists)."""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow
from tests.conftest import golden_model

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8


def _scrambled(m, seed):
    rng = np.random.default_rng(seed)
    mk = m.copy()
    mk.va_deg = m.va_deg + rng.uniform(-120, 120, m.n_bus)
    return mk


def test_oracle_retry_recovers_the_published_solution():
    m, pub = golden_model("case118")
    mk = _scrambled(m, 0)
    plain = oracle.solve(mk, PowerFlowOptions(max_iterations=20).to_c())
    assert plain["status"] == _abi.PF_MAX_ITERATIONS
    r = oracle.solve(mk, PowerFlowOptions(max_iterations=20, retry_from_dc_start=True).to_c())
    assert r["status"] == _abi.PF_CONVERGED and r["iterations"] <= 6
    slack = int(np.nonzero(m.bus_type == 3)[0][0])
    va = r["va_deg"] - r["va_deg"][slack] + pub["va_deg"][slack]
    assert np.max(np.abs(r["vm"] - pub["vm"])) <= pub["vm_tol"]
    assert np.max(np.abs(va - pub["va_deg"])) <= pub["va_tol_deg"]


def test_oracle_retry_leaves_converging_solves_alone():
    m, _ = golden_model("case57")
    a = oracle.solve(m, PowerFlowOptions().to_c())
    b = oracle.solve(m, PowerFlowOptions(retry_from_dc_start=True).to_c())
    assert a["status"] == b["status"] == _abi.PF_CONVERGED
    assert a["iterations"] == b["iterations"]
    assert np.array_equal(a["vm"], b["vm"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["case57", "case118", "case300"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_single_solve_retry_matches_oracle(name, precision):
    m, _ = golden_model(name)
    mk = _scrambled(m, 1)
    opt = PowerFlowOptions(max_iterations=20, retry_from_dc_start=True, precision=precision)
    r = SparseNewtonRaphsonPowerFlow(precision).solve(mk, opt)
    ref = oracle.solve(mk, opt.to_c())
    assert r.status == ref["status"] == _abi.PF_CONVERGED
    assert r.iterations == ref["iterations"]
    assert np.max(np.abs(r.vm - ref["vm"])) <= VM_TOL
    assert np.max(np.abs(np.radians(r.va_deg - ref["va_deg"]))) <= VA_TOL_RAD


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cold_start_screen_retry_matches_oracle(precision):
    m = _scrambled(synthetic.config_grid(0, 0), 2)
    idx = synthetic.outage_set(m, None, 0)[:60]
    opt = PowerFlowOptions(max_iterations=20, retry_from_dc_start=True, per_bus_voltage_limits=True, precision=precision)
    gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), opt, keep_states=True)
    ref = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    assert np.array_equal(gpu["status"], ref["status"])
    assert np.array_equal(gpu["iterations"], ref["iterations"])
    conv = ref["status"] == 0
    assert conv.sum() > 40  # the retry rescues the scrambled starts
    assert np.max(np.abs(gpu["vm"][conv] - ref["vm"][conv])) <= VM_TOL
    assert np.max(np.abs(np.radians(gpu["va_deg"][conv] - ref["va_deg"][conv]))) <= VA_TOL_RAD
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])
    plain = oracle.screen(m, idx, PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True).to_c())
    assert (plain["status"] == 0).sum() < conv.sum()


@pytest.mark.gpu
def test_q_limits_with_retry_match_oracle():
    m, _ = golden_model("case118")
    mk = _scrambled(m, 3)
    opt = PowerFlowOptions(max_iterations=30, retry_from_dc_start=True, enforce_q_limits=True)
    r = SparseNewtonRaphsonPowerFlow("fp64").solve(mk, opt)
    ref = oracle.solve(mk, opt.to_c())
    assert r.status == ref["status"]
    assert r.iterations == ref["iterations"]
    if ref["status"] == _abi.PF_CONVERGED:
        assert np.max(np.abs(r.vm - ref["vm"])) <= VM_TOL
