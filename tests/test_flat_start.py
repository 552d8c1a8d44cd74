"""PowerFlowOptions.FlatStart (``PowerFlow/PowerFlowOptions.cs:95``; start rule ``NewtonShell.cs:463-474``).

The library takes a flat start through the descriptor (its calls refuse the flag): the host wrappers solve the
model's flat-start copy (``GridModel.flat_started``) with the flag cleared. The CPU tests show on the oracle that
the copy solved without the flag is the flagged solve of the original, bit for bit, for single solves (with and
without Q limits and the DC retry) and screens; the GPU tests hold the device path to the oracle's flagged solve.
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow, study_options
from gridsim_b200.model import SLACK
from tests.conftest import assert_states_close, golden_model

CASES = ["case9", "case14", "case57", "case118", "case300"]


def _same(a, b, keys):
    for k in keys:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("study", [False, True])
def test_flat_copy_is_the_flagged_solve(name, study):
    m, _ = golden_model(name)
    opt = study_options() if study else PowerFlowOptions()
    opt = PowerFlowOptions(**{**opt.__dict__, "flat_start": True})
    flagged = oracle.solve(m, opt.to_c())
    copied = oracle.solve(opt.device_model(m), opt.device_c())
    assert flagged["status"] == _abi.PF_CONVERGED
    _same(flagged, copied, ["status", "iterations", "max_mismatch", "vm", "va_deg", "p_inj_mw", "q_inj_mvar"])


def test_flat_start_is_not_vacuous():
    """The stored voltages of the golden cases are near solutions, so a flat start takes more iterations."""
    more = 0
    for name in CASES:
        m, _ = golden_model(name)
        stored = oracle.solve(m, PowerFlowOptions().to_c())
        flat = oracle.solve(m, PowerFlowOptions(flat_start=True).to_c())
        more += flat["iterations"] > stored["iterations"]
    assert more >= 3


@pytest.mark.parametrize("name", ["case14", "case57"])
def test_flat_copy_screen_is_the_flagged_screen(name):
    m, _ = golden_model(name)
    opt = PowerFlowOptions(**{**study_options().__dict__, "flat_start": True})
    idx = m.in_service_branches()
    flagged = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    copied = oracle.screen(opt.device_model(m), idx, opt.device_c(), keep_states=True)
    _same(flagged, copied, ["status", "iterations", "viol_ptr", "viol_kind", "viol_element", "viol_value", "vm",
                            "va_deg", "islanded"])


def test_flat_copy_keeps_reference_buses_and_the_original():
    m = synthetic.config_grid(0, 0)
    f = m.flat_started()
    ref = m.bus_type == SLACK
    assert np.array_equal(f.vm[ref], m.vm[ref]) and np.array_equal(f.va_deg[ref], m.va_deg[ref])
    assert np.all(f.vm[~ref] == 1.0) and np.all(f.va_deg[~ref] == 0.0)
    assert f is not m and not np.shares_memory(f.vm, m.vm)
    o = PowerFlowOptions(flat_start=True)
    assert o.to_c().flat_start == 1 and o.device_c().flat_start == 0
    assert PowerFlowOptions().device_model(m) is m


def test_case9_one_iteration_from_flat_reports_max_iterations():
    """PowerFlowTests.cs:27-36 through the flat-start copy."""
    m, _ = golden_model("case9")
    opt = PowerFlowOptions(max_iterations=1, flat_start=True)
    assert oracle.solve(opt.device_model(m), opt.device_c())["status"] == _abi.PF_MAX_ITERATIONS


@pytest.mark.gpu
@pytest.mark.parametrize("name,precision", [(c, "fp64") for c in CASES] + [(c, "mixed") for c in CASES[:4]])
def test_device_flat_start_matches_oracle(name, precision):
    m, _ = golden_model(name)
    opt = PowerFlowOptions(flat_start=True, precision=precision)
    r = SparseNewtonRaphsonPowerFlow(precision).solve(m, opt)
    ref = oracle.solve(m, opt.to_c())
    assert r.status == ref["status"] == _abi.PF_CONVERGED
    assert np.max(np.abs(r.vm - ref["vm"])) <= 1e-8
    assert np.max(np.abs(np.radians(r.va_deg - ref["va_deg"]))) <= 1e-8


@pytest.mark.gpu
def test_device_flat_start_screen_matches_oracle():
    m, _ = golden_model("case57")
    opt = PowerFlowOptions(flat_start=True)
    idx = m.in_service_branches()
    gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(), opt, keep_states=True)
    ref = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    assert np.array_equal(gpu["status"] == 0, ref["status"] == 0)
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(gpu["viol_kind"], ref["viol_kind"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])
    for j in np.nonzero(ref["status"] == 0)[0]:
        assert_states_close(m, [idx[j]], gpu["vm"][j], gpu["va_deg"][j], ref["vm"][j], ref["va_deg"][j], 1e-8, 1e-8)
