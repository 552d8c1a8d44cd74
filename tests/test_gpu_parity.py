"""Engine vs oracle on the same inputs, through the C ABI (needs a B200).

Parity bar: identical convergence flags; converged voltages within 1e-8 pu and angles within 1e-8 rad
(VM_TOL / VA_TOL_RAD below); identical violation lists (kind, element) with values within 1e-6.
"""
import math

import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow
from tests.conftest import golden_model

pytestmark = pytest.mark.gpu

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8


def _oracle_opts(opt: PowerFlowOptions):
    return opt.to_c()


@pytest.fixture(scope="module")
def grids():
    return {c: synthetic.config_grid(c, 0) for c in (0, 1)}


@pytest.mark.parametrize("name", ["case9", "case14", "case57", "case118", "case300"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_single_solve_matches_oracle(name, precision):
    m, pub = golden_model(name)
    opt = PowerFlowOptions(precision=precision)
    r = SparseNewtonRaphsonPowerFlow(precision).solve(m, opt)
    ref = oracle.solve(m, _oracle_opts(opt))
    assert r.status == ref["status"] == _abi.PF_CONVERGED
    assert r.max_mismatch < 1e-8
    assert np.max(np.abs(r.vm - ref["vm"])) <= VM_TOL
    assert np.max(np.abs(np.radians(r.va_deg - ref["va_deg"]))) <= VA_TOL_RAD
    assert np.max(np.abs(r.p_inj_mw - ref["p_inj_mw"])) < 1e-5
    assert np.max(np.abs(r.loading_percent - ref["loading_pct"])) < 1e-6
    slack = int(np.nonzero(m.bus_type == 3)[0][0])
    va = r.va_deg - r.va_deg[slack] + pub["va_deg"][slack]
    assert np.max(np.abs(r.vm - pub["vm"])) <= pub["vm_tol"]
    assert np.max(np.abs(va - pub["va_deg"])) <= pub["va_tol_deg"]


def _compare_screen(m, idx, opt, precision):
    solver = SparseNewtonRaphsonPowerFlow(precision)
    gpu = ContingencyAnalysis.screen_raw(m, idx, solver, opt, keep_states=True)
    ref = oracle.screen(m, idx, _oracle_opts(opt), keep_states=True)
    assert np.array_equal(gpu["status"] == 0, ref["status"] == 0), "convergence flags differ"
    conv = ref["status"] == 0
    dvm = np.max(np.abs(gpu["vm"][conv] - ref["vm"][conv])) if conv.any() else 0.0
    dva = np.max(np.abs(np.radians(gpu["va_deg"][conv] - ref["va_deg"][conv]))) if conv.any() else 0.0
    assert dvm <= VM_TOL, f"max |dVm| {dvm:.3e}"
    assert dva <= VA_TOL_RAD, f"max |dVa| {dva:.3e} rad"
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"]), "violation counts differ"
    assert np.array_equal(gpu["viol_kind"], ref["viol_kind"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])
    assert np.allclose(gpu["viol_value"], ref["viol_value"], rtol=0, atol=1e-6)
    assert np.allclose(gpu["max_loading_pct"][conv], ref["max_loading_pct"][conv], rtol=0, atol=1e-6)
    assert np.allclose(gpu["min_vm"][conv], ref["min_vm"][conv], rtol=0, atol=VM_TOL)
    return gpu, ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_n1_case118_matches_oracle(precision):
    m, _ = golden_model("case118")
    opt = PowerFlowOptions(max_iterations=100, precision=precision)
    _compare_screen(m, m.in_service_branches(), opt, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_n1_synthetic_120_bus(grids, precision):
    m = grids[0]
    opt = PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True, warm_start_from_base=True,
                           precision=precision)
    idx = synthetic.outage_set(m, None, 0)
    gpu, _ = _compare_screen(m, idx, opt, precision)
    assert gpu["base_status"] == _abi.PF_CONVERGED


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_n1_synthetic_2000_bus(grids, precision):
    m = grids[1]
    opt = PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True, warm_start_from_base=True,
                           precision=precision)
    idx = synthetic.outage_set(m, None, 0)
    _compare_screen(m, idx, opt, precision)


def test_solve_batch_load_scalings(grids):
    m = grids[0]
    sc = synthetic.load_scalings(m, 64, 0) * 0.5 + 0.5
    solver = SparseNewtonRaphsonPowerFlow("mixed")
    out = solver.solve_batch(m, load_scale=sc, options=PowerFlowOptions(precision="mixed"), keep_states=True)
    for k in range(0, 64, 9):
        mk = m.copy()
        mk.pd = m.pd * sc[k]
        mk.qd = m.qd * sc[k]
        ref = oracle.solve(mk)
        assert out["status"][k] == ref["status"]
        if ref["status"] == 0:
            assert np.max(np.abs(out["vm"][k] - ref["vm"])) <= VM_TOL
            assert np.max(np.abs(np.radians(out["va_deg"][k] - ref["va_deg"]))) <= VA_TOL_RAD
