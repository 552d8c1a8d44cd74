"""Voltage-dependent (ZIP) loads: Bus.Zip / ZipLoad (Model/Model.cs:45-90), the mismatch deviation and Jacobian
diagonals of SparseNewtonRaphsonPowerFlow.cs:223-250 (NewtonShell.ZipDeviationPu / ZipJacobianDiagPu :396-413), and the
Q-limit check on the load drawn at the solved voltage (NewtonShell.ApplyQLimits :533-537).

CPU: the oracle pinned on the reference's own ZIP known answers (tests/GridSim.Tests/ZipLoadTests.cs):
  * an explicit constant-power ZIP (0, 0, 1) solves bit for bit as no ZIP (:38-53);
  * a constant-impedance load sags less and draws less than a constant-power one (:55-72);
  * the solved load equals the ZIP polynomial at the solved voltage (:74-88);
and the JSON case reader's ZIP rules (JsonGridLoader.ParseZipValues, IO/Json/JsonGridLoader.cs:395-427).
GPU: the engine against the oracle on ZIP-bearing grids: single solves in both precisions, an N-1 screen, and
Q-limit enforcement under StudyOptions.
"""
import json
import os

import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.model import GridModel, PQ, SLACK, load_case_dir, save_case_dir

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8
CP = (0.0, 0.0, 1.0, 0.0, 0.0, 1.0)


def zip_case(zip_row=None):
    """ZipLoadTests.Case (:20-36): a radial three-bus case with a heavy remote load whose voltage sags."""
    zip_arr = None if zip_row is None else np.array([CP, zip_row, zip_row], np.float64)
    return GridModel(
        name="zip-test", base_mva=100.0, bus_id=np.array([1, 2, 3], np.int32),
        bus_type=np.array([SLACK, PQ, PQ], np.int32), pd=np.array([0.0, 60.0, 90.0]), qd=np.array([0.0, 20.0, 30.0]),
        gs=np.zeros(3), bs=np.zeros(3), vm=np.ones(3), va_deg=np.zeros(3), vmin=np.full(3, np.nan),
        vmax=np.full(3, np.nan), base_kv=np.full(3, 132.0), gen_bus=np.array([0], np.int32), pg=np.zeros(1),
        qg=np.zeros(1), vg=np.ones(1), qmin=np.full(1, -9999.0), qmax=np.full(1, 9999.0),
        gen_in_service=np.ones(1, np.uint8), br_from=np.array([0, 1], np.int32), br_to=np.array([1, 2], np.int32),
        r=np.array([0.02, 0.03]), x=np.array([0.08, 0.10]), b=np.zeros(2), tap=np.ones(2), shift_deg=np.zeros(2),
        rate_a=np.zeros(2), br_in_service=np.ones(2, np.uint8), is_transformer=np.zeros(2, np.uint8), zip=zip_arr)


def with_random_zip(m, seed):
    """The model with a ZIP law on every load bus: Ap U(0, 0.5), Bp U(0, 0.3), Cp the rest (likewise for Q)."""
    rng = np.random.default_rng(seed)
    n = m.n_bus
    z = np.tile(np.array(CP), (n, 1))
    load = (m.pd != 0) | (m.qd != 0)
    for off in (0, 3):
        a = rng.uniform(0.0, 0.5, n)
        bb = rng.uniform(0.0, 0.3, n)
        z[load, off], z[load, off + 1], z[load, off + 2] = a[load], bb[load], (1.0 - a - bb)[load]
    mk = m.copy()
    mk.zip = z
    return mk


def _pmult(z, v):
    return z[0] * v * v + z[1] * v + z[2]


# ---------------------------------------------------------------------------------------------------------- CPU pins

def test_explicit_constant_power_zip_is_bit_for_bit_no_zip():
    plain = oracle.solve(zip_case(None))
    explicit = oracle.solve(zip_case(CP))
    assert plain["status"] == explicit["status"] == _abi.PF_CONVERGED
    assert np.array_equal(plain["vm"], explicit["vm"])
    assert np.array_equal(plain["va_deg"], explicit["va_deg"])


def test_constant_impedance_load_sags_less_and_draws_less():
    cp = oracle.solve(zip_case(None))
    z = oracle.solve(zip_case((1.0, 0.0, 0.0, 1.0, 0.0, 0.0)))
    assert cp["status"] == z["status"] == _abi.PF_CONVERGED
    assert cp["vm"][2] < 1.0
    assert z["vm"][2] > cp["vm"][2]
    assert z["p_inj_mw"][0] < cp["p_inj_mw"][0]  # the slack picks up less load


def test_solved_load_equals_the_zip_polynomial_at_the_solved_voltage():
    zrow = (0.5, 0.3, 0.2, 0.5, 0.3, 0.2)
    r = oracle.solve(zip_case(zrow))
    assert r["status"] == _abi.PF_CONVERGED
    v = r["vm"][2]
    assert abs(r["p_inj_mw"][2] - (-90.0 * _pmult(zrow, v))) < 0.5e-3


def test_json_case_round_trips_zip_and_refuses_bad_blocks(tmp_path):
    m = with_random_zip(synthetic.config_grid(0, 0), 3)
    d = os.path.join(tmp_path, "case")
    save_case_dir(m, d)
    back = load_case_dir(d)
    assert back.zip is not None and np.allclose(back.zip, m.zip, rtol=0, atol=1e-15)
    buses_fn = os.path.join(d, "buses.json")
    with open(buses_fn) as fh:
        buses = json.load(fh)
    k = next(i for i, b in enumerate(buses) if "zip" in b)
    good = dict(buses[k]["zip"])
    for bad, msg in (({**good, "cp": good["cp"] + 0.1}, "sum to"), ({kk: v for kk, v in good.items() if kk != "bq"},
                                                                     "missing coefficient 'bq'")):
        buses[k]["zip"] = bad
        with open(buses_fn, "w") as fh:
            json.dump(buses, fh)
        with pytest.raises(ValueError, match=msg):
            load_case_dir(d)


# ---------------------------------------------------------------------------------------------------------- GPU parity

@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zip_single_solves_match_the_oracle(precision):
    from gridsim_b200.engine import PowerFlowOptions, SparseNewtonRaphsonPowerFlow
    cases = [zip_case((0.5, 0.3, 0.2, 0.5, 0.3, 0.2)), zip_case((1.0, 0.0, 0.0, 1.0, 0.0, 0.0)),
             with_random_zip(synthetic.config_grid(0, 0), 1), with_random_zip(synthetic.config_grid(1, 0), 2)]
    for m in cases:
        opt = PowerFlowOptions(precision=precision)
        r = SparseNewtonRaphsonPowerFlow(precision).solve(m, opt)
        ref = oracle.solve(m, opt.to_c())
        assert r.status == ref["status"] == _abi.PF_CONVERGED, m.name
        assert r.iterations == ref["iterations"], m.name
        assert np.max(np.abs(r.vm - ref["vm"])) <= VM_TOL, m.name
        assert np.max(np.abs(np.radians(r.va_deg - ref["va_deg"]))) <= VA_TOL_RAD, m.name
        assert np.max(np.abs(r.p_inj_mw - ref["p_inj_mw"])) < 1e-5, m.name


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zip_n1_screen_matches_the_oracle(precision):
    from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow
    m = with_random_zip(synthetic.config_grid(1, 0), 4)
    idx = synthetic.outage_set(m, 600, 0)
    opt = PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True, warm_start_from_base=True,
                           precision=precision)
    got = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), opt, keep_states=True)
    ref = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    assert np.array_equal(got["status"], ref["status"])
    assert np.array_equal(got["iterations"], ref["iterations"])
    conv = ref["status"] == _abi.PF_CONVERGED
    assert conv.sum() > 500
    assert np.max(np.abs(got["vm"][conv] - ref["vm"][conv])) <= VM_TOL
    assert np.max(np.abs(np.radians(got["va_deg"][conv] - ref["va_deg"][conv]))) <= VA_TOL_RAD
    assert np.array_equal(got["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(got["viol_element"], ref["viol_element"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["case14", "case57", "case118"])
def test_zip_with_q_limits_matches_the_oracle(name):
    """StudyOptions (Q limits on): a PV bus's generators' output is its injection plus the load drawn at the solved
    voltage, so a ZIP load moves where the limits bind."""
    from gridsim_b200.engine import SparseNewtonRaphsonPowerFlow, study_options
    from tests.conftest import golden_model
    m = with_random_zip(golden_model(name)[0], 5)
    opt = study_options("fp64")
    r = SparseNewtonRaphsonPowerFlow("fp64").solve(m, opt)
    ref = oracle.solve(m, opt.to_c())
    assert r.status == ref["status"]
    assert r.iterations == ref["iterations"]
    if ref["status"] == _abi.PF_CONVERGED:
        assert np.max(np.abs(r.vm - ref["vm"])) <= VM_TOL
        assert np.max(np.abs(np.radians(r.va_deg - ref["va_deg"]))) <= VA_TOL_RAD
