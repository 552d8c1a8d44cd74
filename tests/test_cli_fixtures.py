"""The reference's captured ``gridsim nminus1`` tables (tests/GridSim.Tests/fixtures/cli-stdout/nminus1-*.txt, turned
into ``golden/cli_nminus1.json`` by ``golden/make_golden.py``): for every outage of case9 and case14, the status
(ISLANDED / NO SOLUTION / VIOLATIONxN / base only / secure), the maximum branch and boundary loadings (whole
percent), Vmin and Vmax (three decimals), after netting against the base case, plus the base case's own violations
and the "makes base-case violation(s) worse" notes; and the ``gridsim nminus2`` tables of case9 (top-20 candidate
pairs: the pair count, the count line, the worst pairs in order, the single outages left out of the pairing).

The CLI screens with ContingencyAnalysis.StudyOptions (100 iterations, Q limits, the DC-angle retry) and per-bus
voltage limits unless --global-vlimits (src/GridSim.Cli/Program.cs, RunNMinus1). The same host post-processing
(``ContingencyAnalysis._results`` / ``net_against_base``) reads the oracle's raw screen on the CPU and the engine's on
the GPU, so the first test pins the oracle and the second the CUDA path.
"""
import json
import os

import numpy as np
import pytest

import oracle
from gridsim_b200.engine import ContingencyAnalysis, SparseNewtonRaphsonPowerFlow, study_options
from tests.conftest import GOLDEN, golden_model

with open(os.path.join(GOLDEN, "cli_nminus1.json")) as _fh:
    _ALL = json.load(_fh)
FIXTURES = {k: v for k, v in _ALL.items() if k.startswith("nminus1")}
NM2 = {k: v for k, v in _ALL.items() if k.startswith("nminus2")}


def _status(c):
    """ContingencyStatus (src/GridSim.Cli/Program.cs)."""
    if not c.converged:
        return "ISLANDED" if c.islanded else "NO SOLUTION"
    if not c.secure:
        return f"VIOLATIONx{len(c.violations)}"
    return "base only" if c.pre_existing_violations else "secure"


def _check(fx, model, raw_of):
    idx = model.in_service_branches()
    base = ContingencyAnalysis._results(model, [-1], raw_of(np.array([-1], np.int32)))[0]
    assert base.converged
    assert base.violations == fx["base"]
    rows = ContingencyAnalysis._results(model, idx, raw_of(idx))
    got = {}
    for c in rows:
        c = ContingencyAnalysis.net_against_base(model, c, base)
        got[c.outage] = c
    assert sorted(got) == sorted(r["outage"] for r in fx["rows"])
    for r in fx["rows"]:
        c = got[r["outage"]]
        assert _status(c) == r["status"], r["outage"]
        if "text" in r:
            assert c.violations == [r["text"]], r["outage"]
            continue
        assert f"{c.max_branch_loading_percent:.0f}" == str(r["max_load"]), r["outage"]
        assert f"{c.worst_boundary_loading_percent:.0f}" == str(r["worst_bnd"]), r["outage"]
        assert f"{c.min_vm:.3f}" == r["vmin"], r["outage"]
        assert f"{c.max_vm:.3f}" == r["vmax"], r["outage"]
        if c.pre_existing_violations and not c.violations:
            assert c.worsened_pre_existing_violations == fx["worsened"].get(r["outage"], []), r["outage"]


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_oracle_reproduces_the_cli_table(name):
    fx = FIXTURES[name]
    m, _ = golden_model(fx["case"])
    opt = study_options()
    opt.per_bus_voltage_limits = fx["per_bus_voltage_limits"]
    _check(fx, m, lambda idx: oracle.screen(m, idx, opt.to_c()))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_engine_reproduces_the_cli_table(name, precision):
    fx = FIXTURES[name]
    m, _ = golden_model(fx["case"])
    opt = study_options(precision)
    opt.per_bus_voltage_limits = fx["per_bus_voltage_limits"]
    solver = SparseNewtonRaphsonPowerFlow(precision)
    _check(fx, m, lambda idx: ContingencyAnalysis.screen_raw(m, idx, solver, opt))


def _check_nm2(fx, report):
    res = report.results
    assert len(res) == fx["screened"]
    secure = sum(1 for c in res if c.secure)
    viol = sum(1 for c in res if c.converged and not c.secure)
    isl = sum(1 for c in res if not c.converged and c.islanded)
    assert [len(res), secure, viol, isl] == fx["counts"]
    for r, c in zip(fx["rows"], res):
        assert c.outage == r["outage"]
        assert _status(c) == r["status"]
        if "text" in r:
            assert c.violations == [r["text"]]
    assert [[c.outage, c.violations[0]] for c in report.excluded_single_outages] == fx["excluded"]


@pytest.mark.parametrize("name", sorted(NM2))
def test_oracle_reproduces_the_n_minus_2_table(name):
    fx = NM2[name]
    m, _ = golden_model(fx["case"])
    opt = study_options()
    opt.per_bus_voltage_limits = fx["per_bus_voltage_limits"]
    o = opt.to_c()
    report = ContingencyAnalysis._nk_report(m, fx["k"], lambda idx: oracle.screen(m, idx, o),
                                            lambda sets: oracle.screen_sets(m, sets, o), fx["candidate_count"], False)
    _check_nm2(fx, report)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(NM2))
def test_engine_reproduces_the_n_minus_2_table(name, precision):
    fx = NM2[name]
    m, _ = golden_model(fx["case"])
    opt = study_options(precision)
    opt.per_bus_voltage_limits = fx["per_bus_voltage_limits"]
    report = ContingencyAnalysis.screen_n_minus_k_report(m, fx["k"], SparseNewtonRaphsonPowerFlow(precision), opt,
                                                         candidate_count=fx["candidate_count"])
    _check_nm2(fx, report)
