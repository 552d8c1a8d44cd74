"""Multi-branch outages (gs_nk_screen: ScreenOutageCore over several indices, ContingencyAnalysis.cs:1087-1097) and
the N-k screen around them (ScreenNMinusKReport :378-426).

The device takes a set's branches out of Y by replacing every cell they touch with its value summed without all of
them (shared cells: parallel branches, branches meeting at a bus). GPU results are held to the oracle, which takes the
branches out of a copy of the model: identical statuses, islanding flags and violation lists, converged voltages
within 1e-8 pu and angles within 1e-8 rad (angles of a part left without a reference bus compared as differences within the part: their
common offset is not determined).
"""
import itertools

import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi
from gridsim_b200.engine import (ContingencyAnalysis, EngineError, PowerFlowOptions, SparseNewtonRaphsonPowerFlow,
                                 study_options)
from tests.conftest import assert_states_close, golden_model

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8


def _compare(gpu, ref, m, sets):
    assert np.array_equal(gpu["status"], ref["status"])
    assert np.array_equal(gpu["islanded"], ref["islanded"])
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(gpu["viol_kind"], ref["viol_kind"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])
    for j in np.nonzero(ref["status"] == _abi.PF_CONVERGED)[0]:
        assert_states_close(m, sets[j], gpu["vm"][j], gpu["va_deg"][j], ref["vm"][j], ref["va_deg"][j], VM_TOL,
                            VA_TOL_RAD)


def _parallel_pairs(m):
    """Branch pairs joining the same two buses (their cells coincide)."""
    seen, out = {}, []
    for k in m.in_service_branches():
        key = tuple(sorted((int(m.br_from[k]), int(m.br_to[k]))))
        if key in seen:
            out.append((seen[key], int(k)))
        seen.setdefault(key, int(k))
    return out


def test_oracle_sets_of_one_equal_the_single_screen():
    m, _ = golden_model("case14")
    idx = m.in_service_branches()
    sets = np.full((idx.shape[0], 3), -1, np.int32)
    sets[:, 1] = idx
    opt = study_options().to_c()
    a = oracle.screen(m, idx, opt, keep_states=True)
    b = oracle.screen_sets(m, sets, opt, keep_states=True)
    for key in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "islanded"):
        assert np.array_equal(a[key], b[key]), key
    assert np.array_equal(a["vm"], b["vm"]) and np.array_equal(a["va_deg"], b["va_deg"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["case9", "case14", "case57"])
def test_exhaustive_pairs_match_the_oracle(name, precision):
    """Every pair of in-service branches (N232_case9_n_minus_2_is_bit_identical_to_the_full_solve covers case9's 36),
    under StudyOptions."""
    m, _ = golden_model(name)
    sets = np.array(list(itertools.combinations(m.in_service_branches().tolist(), 2)), np.int32)
    opt = study_options(precision)
    gpu = ContingencyAnalysis.screen_sets_raw(m, sets, SparseNewtonRaphsonPowerFlow(precision), opt, keep_states=True)
    ref = oracle.screen_sets(m, sets, opt.to_c(), keep_states=True)
    _compare(gpu, ref, m, sets)
    assert (gpu["status"] == _abi.PF_UNSOLVABLE_PART).any() or name != "case9"


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_case118_pairs_triples_and_parallel_branches(precision):
    """case118: 3,000 sampled pairs, the parallel pairs (shared cells), triples and quadruples around shared buses,
    rows with -1 padding (an N-1 outage and the intact grid in the same call)."""
    m, _ = golden_model("case118")
    live = m.in_service_branches()
    rng = np.random.default_rng(11)
    rows = [list(rng.choice(live, 2, replace=False)) for _ in range(3000)]
    par = _parallel_pairs(m)
    assert par
    rows += [list(p) for p in par]
    rows += [list(p) + [int(rng.choice(live))] for p in par if True]
    for b in rng.choice(m.n_bus, 40, replace=False):  # every branch at a bus, up to four
        at = [int(k) for k in live if m.br_from[k] == b or m.br_to[k] == b][:4]
        if len(at) >= 2:
            rows.append(at)
    rows.append([int(live[5])])
    rows.append([])
    width = 4
    sets = np.full((len(rows), width), -1, np.int32)
    for j, r in enumerate(rows):
        r = list(dict.fromkeys(int(x) for x in r))[:width]
        sets[j, :len(r)] = r
    opt = PowerFlowOptions(precision=precision, warm_start_from_base=True, per_bus_voltage_limits=True)
    gpu = ContingencyAnalysis.screen_sets_raw(m, sets, SparseNewtonRaphsonPowerFlow(precision), opt, keep_states=True)
    ref = oracle.screen_sets(m, sets, opt.to_c(), keep_states=True)
    _compare(gpu, ref, m, sets)


@pytest.mark.gpu
def test_n_minus_2_report_matches_the_oracle_pipeline():
    m, _ = golden_model("case118")
    opt = study_options("mixed")
    o = opt.to_c()
    rep = ContingencyAnalysis.screen_n_minus_k_report(m, 2, SparseNewtonRaphsonPowerFlow("mixed"), opt,
                                                      candidate_count=30)
    ref = ContingencyAnalysis._nk_report(m, 2, lambda idx: oracle.screen(m, idx, o),
                                         lambda sets: oracle.screen_sets(m, sets, o), 30, False)
    assert len(rep.results) == len(ref.results) == 435
    assert [c.outage for c in rep.excluded_single_outages] == [c.outage for c in ref.excluded_single_outages]
    assert sorted(c.outage for c in rep.results) == sorted(c.outage for c in ref.results)
    by = {c.outage: c for c in ref.results}
    for c in rep.results:
        r = by[c.outage]
        assert (c.converged, c.islanded, c.violations) == (r.converged, r.islanded, r.violations), c.outage


@pytest.mark.gpu
def test_bad_sets_are_refused():
    m, _ = golden_model("case14")
    solver = SparseNewtonRaphsonPowerFlow()
    opt = PowerFlowOptions()
    with pytest.raises(EngineError):
        ContingencyAnalysis.screen_sets_raw(m, np.array([[3, 3]], np.int32), solver, opt)   # a branch twice
    with pytest.raises(EngineError):
        ContingencyAnalysis.screen_sets_raw(m, np.arange(17, dtype=np.int32)[None, :], solver, opt)  # 17 branches
    with pytest.raises(EngineError):
        ContingencyAnalysis.screen_sets_raw(m, np.array([[0, m.n_branch]], np.int32), solver, opt)  # no such branch
