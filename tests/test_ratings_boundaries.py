"""Post-fault ratings, transmission boundaries and islanding in the N-1 screen.

* PostFaultRating B / C (PowerFlowOptions.cs:162-170): an outage state's branch loadings are judged against RateB /
  RateC, RateA where that rating is 0; the base case always against RateA (ContingencyAnalysis.cs:1150-1159,
  PostFaultLoadingPercent :1273-1284).
* Boundaries (BoundaryAnalysis.EvaluateAfterOutage, Analysis/BoundaryAnalysis.cs:43-68): the signed sum of the members'
  from-end MW against the limit (0 = none), BoundaryOverload entries between the branch and voltage entries, the
  worst boundary loading per outage.
* Outages that split the network: "islanded" when not converged, and the provably unsolvable ones reported without a
  solve (ScreenStateCore :1118-1127).

The CPU tests pin the oracle's classification against numbers computed here from its own solved state; the GPU tests
hold the engine to the oracle: identical statuses, islanding flags and violation lists (kind, element), loadings within
LOAD_TOL percent.
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow
from tests.conftest import golden_model

LOAD_TOL = 1e-6  # percent


def _rated_grid():
    """The 120-bus synthetic grid with RateB on every other branch (0 on the rest: RateA applies), RateC on all,
    named branches and four boundaries, one of them without a limit."""
    m = synthetic.config_grid(0, 0)
    nb = m.n_branch
    m.rate_b = np.where(np.arange(nb) % 2 == 0, 0.55 * m.rate_a, 0.0)
    m.rate_c = 0.8 * m.rate_a
    m.br_name = [f"L{k}" for k in range(nb)]
    base = oracle.solve(m)
    pf = base["sf_mva"][0::2]
    # cut sets: the branches leaving the first 10, 30 and 60 buses (by position), signed out of the set
    bnds = []
    for q, (size, frac) in enumerate([(10, 0.9), (30, 1.05), (60, 0.7)]):
        inside = np.zeros(m.n_bus, bool)
        inside[:size] = True
        mem, flow = [], 0.0
        for k in range(nb):
            a, b = inside[m.br_from[k]], inside[m.br_to[k]]
            if a != b:
                d = 1 if a else -1
                mem.append((f"L{k}", d))
                flow += d * pf[k]
        bnds.append((f"cut{q}", round(abs(flow) * frac, 1), mem))
    bnds.append(("unlimited", 0.0, bnds[0][2]))
    m.boundaries = bnds
    return m


def _compare(gpu, ref):
    assert np.array_equal(gpu["status"], ref["status"])
    assert np.array_equal(gpu["islanded"], ref["islanded"])
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(gpu["viol_kind"], ref["viol_kind"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])
    load = np.isin(ref["viol_kind"], [_abi.VIOL_BRANCH_OVERLOAD, _abi.VIOL_BOUNDARY_OVERLOAD])
    assert np.max(np.abs(gpu["viol_value"][load] - ref["viol_value"][load]), initial=0) <= LOAD_TOL
    assert np.max(np.abs(gpu["max_loading_pct"] - ref["max_loading_pct"])) <= LOAD_TOL
    assert np.max(np.abs(gpu["worst_boundary_pct"] - ref["worst_boundary_pct"])) <= LOAD_TOL


def test_oracle_boundary_and_rating_arithmetic():
    """The oracle's screen of one outage against loadings recomputed here from its own solved state."""
    m = _rated_grid()
    k = int(synthetic.outage_set(m, 1, 3)[0])
    for rating in ("A", "B", "C"):
        opt = PowerFlowOptions(post_fault_rating=rating)
        r = oracle.screen(m, [k], opt.to_c(), keep_states=True)
        assert r["status"][0] == _abi.PF_CONVERGED
        mk = m.copy()
        mk.br_in_service = m.br_in_service.copy()
        mk.br_in_service[k] = 0
        mk.vm, mk.va_deg = r["vm"][0], r["va_deg"][0]
        s = oracle.solve(mk, PowerFlowOptions(max_iterations=0).to_c())  # line flows of that state
        sf = s["sf_mva"][0::2] + 1j * s["sf_mva"][1::2]
        st = s["st_mva"][0::2] + 1j * s["st_mva"][1::2]
        mva = np.maximum(np.abs(sf), np.abs(st))
        rate = m.rate_a.copy()
        if rating != "A":
            rx = m.rate_b if rating == "B" else m.rate_c
            rate = np.where(rx > 0, rx, m.rate_a)
        load = np.where(rate > 0, mva / np.where(rate > 0, rate, 1) * 100, 0)
        load[k] = 0
        assert abs(r["max_loading_pct"][0] - load.max()) < 1e-9
        a, b = r["viol_ptr"][0], r["viol_ptr"][1]
        kinds, els = r["viol_kind"][a:b], r["viol_element"][a:b]
        assert sorted(els[kinds == _abi.VIOL_BRANCH_OVERLOAD].tolist()) == np.nonzero(load > 100)[0].tolist()
        ptr, br, dr, lim = m.boundary_members()
        worst, over = 0.0, []
        for q in range(len(lim)):
            flow = sum(dr[e] * sf[br[e]].real for e in range(ptr[q], ptr[q + 1]) if br[e] != k)
            pct = abs(flow) / lim[q] * 100 if lim[q] > 0 else 0.0
            worst = max(worst, pct)
            if lim[q] > 0 and abs(flow) > lim[q]:
                over.append(q)
        assert abs(r["worst_boundary_pct"][0] - worst) < 1e-9
        assert els[kinds == _abi.VIOL_BOUNDARY_OVERLOAD].tolist() == over
        # the order of the list: branches, then boundaries, then buses
        order = [{_abi.VIOL_BRANCH_OVERLOAD: 0, _abi.VIOL_BOUNDARY_OVERLOAD: 1}.get(int(x), 2) for x in kinds]
        assert order == sorted(order)


def test_boundary_names_must_resolve_to_one_branch():
    m = _rated_grid()
    m.br_name[5] = m.br_name[6]
    m.boundaries = [("b", 10.0, [(m.br_name[6], 1)])]
    with pytest.raises(ValueError, match="2 branches share"):
        m.desc()
    m.boundaries = [("b", 10.0, [("nothing", 1)])]
    with pytest.raises(ValueError, match="matches no branch"):
        m.desc()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("rating", ["A", "B", "C"])
def test_ratings_and_boundaries_match_the_oracle(precision, rating):
    m = _rated_grid()
    idx = np.concatenate([[-1], synthetic.outage_set(m, None, 0)]).astype(np.int32)
    opt = PowerFlowOptions(precision=precision, post_fault_rating=rating, warm_start_from_base=True,
                           per_bus_voltage_limits=True)
    gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), opt)
    ref = oracle.screen(m, idx, opt.to_c())
    _compare(gpu, ref)
    kinds = set(ref["viol_kind"].tolist())
    assert _abi.VIOL_BRANCH_OVERLOAD in kinds and _abi.VIOL_BOUNDARY_OVERLOAD in kinds
    # the base case (position 0) is judged against RateA whatever the option
    if rating != "A":
        base = ContingencyAnalysis.screen_raw(m, idx[:1], SparseNewtonRaphsonPowerFlow(precision),
                                              PowerFlowOptions(precision=precision))
        assert abs(gpu["max_loading_pct"][0] - base["max_loading_pct"][0]) <= LOAD_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_islanded_and_unsolvable_outages(precision):
    """case9 and case118 under StudyOptions: every in-service branch, the provably unsolvable outages interleaved
    with solved ones and the intact grid; the same statuses, flags and violation CSR as the oracle."""
    for name in ("case9", "case118"):
        m, _ = golden_model(name)
        idx = np.concatenate([m.in_service_branches(), [-1]]).astype(np.int32)
        opt = PowerFlowOptions(max_iterations=100, enforce_q_limits=True, retry_from_dc_start=True,
                               precision=precision)
        gpu = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), opt)
        ref = oracle.screen(m, idx, opt.to_c())
        _compare(gpu, ref)
        un = gpu["status"] == _abi.PF_UNSOLVABLE_PART
        assert un.sum() == {"case9": 3, "case118": 8}[name]
        assert gpu["islanded"][un].all()
        assert (gpu["iterations"][un] == 0).all()
        res = ContingencyAnalysis._results(m, idx, gpu)
        assert all(r.violations == ["islanded"] for r, u in zip(res, un) if u)
