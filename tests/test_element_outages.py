"""Generator and bus outages (gs_element_screen: ContingencyAnalysis.ScreenElementOutages / ScreenElementOutage,
Analysis/ContingencyAnalysis.cs:1309-1437, with the reference-bus dispatch).

The oracle builds each outage's reduced model as the reference does (the unit, or the bus with its branches, units and
load, taken out; a PV bus left without units solved as PQ; ReelectReference when the outage takes the reference's last
unit or the reference bus) and solves it. The device keeps the grid's size: every bus has P and Q rows, a removed bus
and a reference keep identity rows, and the per-system bus types and lost output are overrides. GPU results are held
to the oracle: identical statuses, islanding flags and violation lists, converged voltages within 1e-8 pu and angles
within 1e-8 rad on the buses that remain.

The three-bus cases are those of the reference's ContingencyTypesAndRatingsTests.cs:164-237.
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow, study_options
from gridsim_b200.model import PQ, PV, SLACK, GridModel
from tests.conftest import assert_states_close, golden_model

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8


def three_bus(units=(40.0, 60.0)):
    """ThreeBus (ContingencyTypesAndRatingsTests.cs:164-171): bus 1 the reference, bus 2 PV, bus 3 a 100 MW load."""
    ng = len(units)
    return GridModel(
        name="three-bus", base_mva=100.0, bus_id=np.array([1, 2, 3], np.int32),
        bus_type=np.array([SLACK, PV, PQ], np.int32), pd=np.array([0.0, 0.0, 100.0]), qd=np.array([0.0, 0.0, 20.0]),
        gs=np.zeros(3), bs=np.zeros(3), vm=np.ones(3), va_deg=np.zeros(3), vmin=np.full(3, np.nan),
        vmax=np.full(3, np.nan), base_kv=np.full(3, 132.0), gen_bus=np.arange(ng, dtype=np.int32),
        pg=np.array(units, float), qg=np.zeros(ng), vg=np.ones(ng), qmin=np.full(ng, -9999.0),
        qmax=np.full(ng, 9999.0), gen_in_service=np.ones(ng, np.uint8), br_from=np.array([0, 1, 0], np.int32),
        br_to=np.array([2, 2, 1], np.int32), r=np.full(3, 0.01), x=np.full(3, 0.1), b=np.zeros(3), tap=np.ones(3),
        shift_deg=np.zeros(3), rate_a=np.full(3, 150.0), br_in_service=np.ones(3, np.uint8),
        is_transformer=np.zeros(3, np.uint8))


def _all_elements(m):
    on = np.nonzero(m.gen_in_service)[0]
    kinds = np.concatenate([np.zeros(m.n_branch), np.ones(len(on)), np.full(m.n_bus, 2)]).astype(np.int32)
    idx = np.concatenate([np.arange(m.n_branch), on, np.arange(m.n_bus)]).astype(np.int32)
    return kinds, idx


def test_oracle_three_bus_cases():
    m = three_bus()
    opt = PowerFlowOptions().to_c()
    r = oracle.screen_elements(m, [1, 1, 2], [1, 0, 0], opt, keep_states=True)
    assert (r["status"] == _abi.PF_CONVERGED).all()  # G2 out; G1 out (the reference moves); bus 1 out (likewise)
    # the G2 outage is the model without G2, solved
    without = m.copy()
    without.gen_in_service = np.array([1, 0], np.uint8)
    pf = oracle.solve(without, opt)
    assert r["min_vm"][0] == np.min(pf["vm"])
    # a one-unit network has nothing left to take over the reference
    lone = oracle.screen_elements(three_bus((40.0,)), [1], [0], opt)
    assert lone["status"][0] == _abi.PF_UNSOLVABLE_PART and not lone["islanded"][0]


def test_oracle_branch_elements_equal_the_branch_screen():
    m, _ = golden_model("case14")
    idx = m.in_service_branches()
    opt = study_options().to_c()
    a = oracle.screen(m, idx, opt)
    b = oracle.screen_elements(m, np.zeros(len(idx), np.int32), idx, opt)
    for key in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "islanded"):
        assert np.array_equal(a[key], b[key]), key


def _compare(gpu, ref, m, kinds, idx):
    assert np.array_equal(gpu["status"], ref["status"])
    assert np.array_equal(gpu["islanded"], ref["islanded"])
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(gpu["viol_kind"], ref["viol_kind"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])
    conv = ref["status"] == _abi.PF_CONVERGED
    for j in np.nonzero(conv)[0]:
        if kinds[j] == 0:
            removed, bus = [idx[j]], -1
        elif kinds[j] == 2:  # a removed bus has no state in the reduced model
            removed = [k for k in range(m.n_branch) if idx[j] in (m.br_from[k], m.br_to[k])]
            bus = idx[j]
        else:
            removed, bus = [], -1
        assert_states_close(m, removed, gpu["vm"][j], gpu["va_deg"][j], ref["vm"][j], ref["va_deg"][j], VM_TOL,
                            VA_TOL_RAD, removed_bus=bus)
    assert np.max(np.abs(gpu["min_vm"][conv] - ref["min_vm"][conv]), initial=0) <= VM_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["case9", "case14", "case57", "case118"])
def test_every_element_outage_matches_the_oracle(name, precision):
    m, _ = golden_model(name)
    kinds, idx = _all_elements(m)
    solver = SparseNewtonRaphsonPowerFlow(precision)
    for opt in (study_options(precision),
                PowerFlowOptions(precision=precision, warm_start_from_base=True, per_bus_voltage_limits=True)):
        gpu = ContingencyAnalysis.screen_elements_raw(m, kinds, idx, solver, opt, keep_states=True)
        ref = oracle.screen_elements(m, kinds, idx, opt.to_c(), keep_states=True)
        _compare(gpu, ref, m, kinds, idx)


@pytest.mark.gpu
def test_three_bus_labels_notes_and_lost_output():
    m = three_bus()
    res = ContingencyAnalysis.screen_element_outages(m, ContingencyAnalysis.single_outages(m, True, True, True))
    assert len(res) == 3 + 2 + 3
    g2, g1 = res[4], res[3]
    assert g2.converged and g2.outage == "gen 1 at bus 2" and g2.lost_generation_mw == 60.0 and g2.note is None
    assert g1.converged and g1.note == "reference moved from bus 1 to bus 2" and g1.lost_generation_mw == 40.0
    b1 = res[5]
    assert b1.converged and b1.outage == "bus 1" and b1.lost_generation_mw == 40.0
    assert b1.note == "reference moved from bus 1 to bus 2"
    b3 = res[7]
    assert b3.lost_load_mw == 100.0
    lone = ContingencyAnalysis.screen_element_outages(three_bus((40.0,)), [(1, 0)])[0]
    assert not lone.converged and "no in-service unit" in lone.note
