"""Generator and bus outages with their lost power shared by governor droop or inertia (OutageDispatch,
``ContingencyAnalysis.cs:120-129``; ShareLostPower :1509-1579; ParticipationWeights :1588-1645).

CPU: the oracle's restatement is pinned on the reference's own known answers (``B3GovernorsDynamicDataTests.N124.cs``,
``PostRc3BatchFTests.cs:64-101``, ``MatpowerInvertedLimitsTests.cs:74-90``); the host's independent restatement
(``engine.share_lost_power``) equals the oracle's bit for bit; and, with the oracle as the solver, the element
outage of the host's moved model (units shared, reference re-elected) under the reference-bus dispatch is the
shared-dispatch outage, bit for bit, for every generator and bus of the golden cases. That is the premise of the
device path, which solves each shared outage as the element outage of its moved model. GPU: the device against
the oracle.
"""
import math

import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi
from gridsim_b200.engine import (ContingencyAnalysis, PowerFlowOptions, SparseNewtonRaphsonPowerFlow,
                                 _shared_outage, share_lost_power)
from gridsim_b200.model import PQ, PV, SLACK, GridModel
from tests.conftest import assert_states_close, golden_model

INF = math.inf


def make_model(buses, gens, branches, base=100.0):
    """buses: (id, type, Pd, Qd); gens: dicts (bus id, pg, pmax, mbase, h, and optionally pmin, type, pf_only);
    branches: (from id, to id, r, x, RateA)."""
    pos = {b[0]: i for i, b in enumerate(buses)}
    n, ng, nb = len(buses), len(gens), len(branches)
    f = lambda v: np.array(v, np.float64)  # noqa: E731
    return GridModel(
        name="hand", base_mva=base, bus_id=np.array([b[0] for b in buses], np.int32),
        bus_type=np.array([b[1] for b in buses], np.int32), pd=f([b[2] for b in buses]), qd=f([b[3] for b in buses]),
        gs=np.zeros(n), bs=np.zeros(n), vm=np.ones(n), va_deg=np.zeros(n), vmin=np.full(n, np.nan),
        vmax=np.full(n, np.nan), base_kv=np.full(n, 132.0),
        gen_bus=np.array([pos[g["bus"]] for g in gens], np.int32), pg=f([g["pg"] for g in gens]), qg=np.zeros(ng),
        vg=np.ones(ng), qmin=np.full(ng, -INF), qmax=np.full(ng, INF), gen_in_service=np.ones(ng, np.uint8),
        br_from=np.array([pos[b[0]] for b in branches], np.int32), br_to=np.array([pos[b[1]] for b in branches], np.int32),
        r=f([b[2] for b in branches]), x=f([b[3] for b in branches]), b=np.zeros(nb), tap=np.ones(nb),
        shift_deg=np.zeros(nb), rate_a=f([b[4] for b in branches]), br_in_service=np.ones(nb, np.uint8),
        is_transformer=np.zeros(nb, np.uint8),
        pmin=f([g.get("pmin", 0.0) for g in gens]), pmax=f([g["pmax"] for g in gens]),
        mbase=f([g["mbase"] for g in gens]), inertia_h=f([g["h"] for g in gens]),
        gen_type=[g.get("type", "ccgt") for g in gens], pf_only=np.array([g.get("pf_only", 0) for g in gens], np.uint8),
        converter=np.full(ng, -1, np.int8))


def n124(g3_pmax=400.0, islands=1):
    """The four-bus model of B3GovernorsDynamicDataTests.N124.cs:17-36 (islands=2: PostRc3BatchFTests.cs:66-85)."""
    buses, gens, brs = [], [], []
    for off in ((0, 10) if islands == 2 else (0,)):
        buses += [(1 + off, SLACK, 0, 0), (2 + off, PV, 0, 0), (3 + off, PQ, 150, 30), (4 + off, PV, 0, 0)]
        gens += [dict(bus=1 + off, pg=40, pmax=200, mbase=100, h=5), dict(bus=2 + off, pg=60, pmax=200, mbase=100, h=4),
                 dict(bus=4 + off, pg=50, pmax=g3_pmax, mbase=300, h=2)]
        brs += [(1 + off, 3 + off, 0.01, 0.1, 250), (2 + off, 3 + off, 0.01, 0.1, 250),
                (1 + off, 2 + off, 0.01, 0.1, 250), (4 + off, 3 + off, 0.01, 0.1, 250)]
    return make_model(buses, gens, brs)


def without(m, unit, **pg):
    r = m.copy()
    r.gen_in_service[unit] = 0
    for k, v in pg.items():
        r.pg[int(k[1:])] = v
    return r


def min_vm(m):
    r = oracle.solve(m)
    assert r["status"] == _abi.PF_CONVERGED
    return float(np.min(r["vm"]))


def gen_outage(m, unit, dispatch):
    return oracle.screen_elements(m, [1], [unit], PowerFlowOptions().to_c(), dispatch=dispatch)


# ---- the oracle against the reference's known answers ------------------------------------------------------
def test_n124_the_default_is_the_reference_bus_screen():
    m = n124()
    r = gen_outage(m, 1, "reference")
    assert r["status"][0] == _abi.PF_CONVERGED and r["notes"] == [None]
    assert r["min_vm"][0] == min_vm(without(m, 1))   # the model without G2 solved directly, bit for bit


def test_n124_governor_droop_shares_by_machine_base():
    m = n124()
    r = gen_outage(m, 1, "droop")
    assert r["status"][0] == _abi.PF_CONVERGED
    assert r["notes"] == ["lost 60.0 MW shared by governor droop over 2 unit(s)"]
    assert r["min_vm"][0] == min_vm(without(m, 1, g0=55.0, g2=95.0))


def test_n124_a_unit_at_its_limit_passes_the_rest_on():
    m = n124(g3_pmax=70.0)
    r = gen_outage(m, 1, "droop")
    assert r["notes"] == ["lost 60.0 MW shared by governor droop over 2 unit(s), 1 at a limit"]
    assert r["min_vm"][0] == min_vm(without(m, 1, g0=80.0, g2=70.0))


def test_n124_inertia_shares_by_stored_energy():
    pg, note = oracle.share_lost_power(without(n124(), 1), 60.0, "inertia")
    assert abs(pg[0] - (40.0 + 60.0 * 500.0 / 1100.0)) < 1e-12
    assert abs(pg[2] - (50.0 + 60.0 * 600.0 / 1100.0)) < 1e-12
    assert note == "lost 60.0 MW shared by inertia over 2 unit(s)"


def converters_model():
    """B3GovernorsDynamicDataTests.N124.cs:100-112: a synchronous unit, a wind plant and a power-flow-only unit."""
    return make_model([(1, SLACK, 0, 0), (2, PQ, 100, 0)],
                      [dict(bus=1, pg=30, pmax=50, mbase=100, h=4), dict(bus=2, pg=20, pmax=200, mbase=400, h=0,
                                                                        type="wind-onshore"),
                       dict(bus=2, pg=10, pmax=200, mbase=400, h=0, pf_only=1)],
                      [(1, 2, 0.01, 0.1, 0)])


def test_converters_and_power_flow_only_units_take_no_share():
    m = converters_model()
    pg, note = oracle.share_lost_power(m, 50.0, "droop")
    assert list(pg) == [50.0, 20.0, 10.0]
    assert note == ("lost 50.0 MW shared by governor droop over 1 unit(s), 1 at a limit; "
                    "30.0 MW beyond their headroom left to the reference")
    pg, note = oracle.share_lost_power(m, -10.0, "droop")
    assert pg[0] == 20.0 and note == "surplus 10.0 MW shared by governor droop over 1 unit(s)"
    with pytest.raises(ValueError):
        oracle.share_lost_power(m, math.nan, "inertia")
    with pytest.raises(ValueError):
        oracle.share_lost_power(m, 5.0, "reference")


def test_lost_power_is_shared_only_inside_the_island_that_lost_it():
    m = n124(islands=2)
    reduced = without(m, 1)
    pg, note = oracle.share_lost_power(reduced, 60.0, "droop", island_buses=[1])   # bus 2 is position 1
    assert abs(pg[0] - (40.0 + 60.0 * 100.0 / 400.0)) < 1e-12
    assert abs(pg[2] - (50.0 + 60.0 * 300.0 / 400.0)) < 1e-12
    assert list(pg[3:]) == list(reduced.pg[3:])
    assert note == "lost 60.0 MW shared by governor droop over 2 unit(s)"
    assert gen_outage(m, 1, "droop")["notes"] == [note]


def crossed_model():
    """MatpowerInvertedLimitsTests.cs:21-39: unit 1 (at bus 2) has PMIN 80 above PMAX 50."""
    m = make_model([(1, SLACK, 0, 0), (2, PV, 0, 0), (3, PQ, 90, 30)],
                   [dict(bus=1, pg=20, pmax=300, pmin=0, mbase=100, h=0),
                    dict(bus=2, pg=40, pmax=50, pmin=80, mbase=100, h=0)],
                   [(1, 2, 0.01, 0.1, 250), (2, 3, 0.01, 0.1, 250), (1, 3, 0.02, 0.2, 250)])
    m.vg[:] = [1.02, 1.01]
    return m


def test_a_crossed_active_power_range_is_refused():
    m = crossed_model()
    with pytest.raises(RuntimeError):
        gen_outage(m, 0, "droop")
    with pytest.raises(ValueError, match="Pmin 80 MW above Pmax 50 MW"):
        _shared_outage(m, 1, 0, "droop")
    assert gen_outage(m, 0, "reference")["notes"] == [None]   # the reference bus takes it: nothing to refuse


# ---- the host's restatement against the oracle's ---------------------------------------------------------
def _with_machines(name, seed):
    m, _ = golden_model(name)
    rng = np.random.default_rng(seed)
    m.inertia_h = rng.uniform(0.0, 8.0, m.n_gen).round(2)
    m.inertia_h[rng.random(m.n_gen) < 0.2] = 0.0
    # tight headroom on some units, so that units reach their limits and the water filling runs again
    m.pmax = np.where(rng.random(m.n_gen) < 0.4, m.pg + rng.uniform(0.0, 15.0, m.n_gen), m.pmax)
    m.pmin = np.minimum(m.pmin, m.pg)
    return m


@pytest.mark.parametrize("name", ["case14", "case57", "case118"])
@pytest.mark.parametrize("dispatch", ["droop", "inertia"])
def test_host_sharing_is_the_oracle_sharing(name, dispatch):
    m = _with_machines(name, 7)
    on = np.nonzero(m.gen_in_service)[0]
    for g in on:
        units = [int(u) for u in on if u != g]
        bus = int(m.gen_bus[g])
        for lost in (float(m.pg[g]), -25.0, 400.0):
            pg_h, note_h = share_lost_power(m, units, m.bus_type, lost, dispatch, [bus])
            pg_o, note_o = oracle.share_lost_power(without(m, int(g)), lost, dispatch, island_buses=[bus])
            assert note_h == note_o
            assert np.array_equal(pg_h, pg_o[units]), (g, lost)


def _element_outages(m):
    on = np.nonzero(m.gen_in_service)[0]
    kinds = [1] * len(on) + [2] * m.n_bus
    idx = [int(g) for g in on] + list(range(m.n_bus))
    return np.array(kinds, np.int32), np.array(idx, np.int32)


@pytest.mark.parametrize("name", ["case9", "case14", "case57"])
@pytest.mark.parametrize("dispatch", ["droop", "inertia"])
def test_moved_model_outage_is_the_shared_outage(name, dispatch):
    """The device path's premise, with the oracle as the solver."""
    m = _with_machines(name, 11)
    kinds, idx = _element_outages(m)
    opt = PowerFlowOptions().to_c()
    shared = oracle.screen_elements(m, kinds, idx, opt, keep_states=True, dispatch=dispatch)
    plain = oracle.screen_elements(m, kinds, idx, opt, keep_states=True)
    moved_any = 0
    for j in range(len(kinds)):
        plan = _shared_outage(m, int(kinds[j]), int(idx[j]), dispatch)
        if plan is None:
            assert shared["notes"][j] is None
            continue
        moved, note = plan
        assert note == shared["notes"][j]
        src = plain if moved is None else oracle.screen_elements(moved, kinds[j:j + 1], idx[j:j + 1], opt,
                                                                 keep_states=True)
        row = j if moved is None else 0
        moved_any += moved is not None
        for key in ("status", "iterations", "max_mismatch", "min_vm", "max_vm", "max_loading_pct", "islanded"):
            assert shared[key][j] == src[key][row], (j, key)
        a, b = shared["viol_ptr"][j], shared["viol_ptr"][j + 1]
        c, d = src["viol_ptr"][row], src["viol_ptr"][row + 1]
        for key in ("viol_kind", "viol_element", "viol_value"):
            assert np.array_equal(shared[key][a:b], src[key][c:d]), (j, key)
        assert np.array_equal(shared["vm"][j], src["vm"][row]) and np.array_equal(shared["va_deg"][j], src["va_deg"][row])
    assert moved_any > 0


def test_reference_move_then_sharing_note():
    """An outage of the reference's last unit: the reference moves first, then the rest share (:1366-1374)."""
    m = n124()
    kinds, idx = np.array([1], np.int32), np.array([0], np.int32)
    r = oracle.screen_elements(m, kinds, idx, PowerFlowOptions().to_c(), dispatch="droop")
    moved, note = _shared_outage(m, 1, 0, "droop")
    assert note == r["notes"][0]
    assert moved.bus_type[0] == PQ and moved.bus_type[1] == SLACK   # G2 (60 MW) is the largest unit left
    assert r["status"][0] == _abi.PF_CONVERGED


# ---- the device against the oracle ---------------------------------------------------------------------------
def _compare(m, kinds, idx, dispatch):
    solver = SparseNewtonRaphsonPowerFlow()
    opt = PowerFlowOptions()
    gpu = ContingencyAnalysis.screen_elements_raw(m, kinds, idx, solver, opt, keep_states=True, dispatch=dispatch)
    ref = oracle.screen_elements(m, kinds, idx, opt.to_c(), keep_states=True, dispatch=dispatch)
    assert gpu["share_notes"] == ref["notes"]
    assert np.array_equal(gpu["status"] == 0, ref["status"] == 0)
    assert np.array_equal(gpu["islanded"], ref["islanded"])
    assert np.array_equal(gpu["viol_ptr"], ref["viol_ptr"])
    assert np.array_equal(gpu["viol_kind"], ref["viol_kind"])
    assert np.array_equal(gpu["viol_element"], ref["viol_element"])
    for j in np.nonzero(ref["status"] == 0)[0]:
        removed = int(idx[j]) if kinds[j] == 2 else -1
        cut = [k for k in range(m.n_branch) if removed in (int(m.br_from[k]), int(m.br_to[k]))] if removed >= 0 else []
        assert_states_close(m, cut, gpu["vm"][j], gpu["va_deg"][j], ref["vm"][j], ref["va_deg"][j], 1e-8, 1e-8,
                            removed_bus=removed)


@pytest.mark.gpu
@pytest.mark.parametrize("dispatch", ["droop", "inertia"])
def test_device_n124(dispatch):
    m = n124(g3_pmax=70.0)
    _compare(m, np.array([1, 1, 1, 2, 2], np.int32), np.array([0, 1, 2, 1, 2], np.int32), dispatch)


@pytest.mark.gpu
@pytest.mark.parametrize("name,dispatch", [("case14", "droop"), ("case57", "droop"), ("case57", "inertia")])
def test_device_shared_outages_match_oracle(name, dispatch):
    m = _with_machines(name, 11)
    kinds, idx = _element_outages(m)
    _compare(m, kinds, idx, dispatch)


@pytest.mark.gpu
def test_device_shared_results_carry_the_notes():
    m = n124()
    res = ContingencyAnalysis.screen_element_outages(m, [(1, 0), (1, 1)], dispatch="droop")
    assert res[0].note.startswith("reference moved from bus 1 to bus 2; lost 40.0 MW shared by governor droop")
    assert res[1].note == "lost 60.0 MW shared by governor droop over 2 unit(s)"
    assert res[1].lost_generation_mw == 60.0 and res[1].converged


# ---- host logic without a device -------------------------------------------------------------------------------
def test_share_lost_power_edge_cases():
    m = converters_model()
    units = [0, 1, 2]
    pg, note = share_lost_power(m, units, m.bus_type, 0.0, "inertia")
    assert list(pg) == [30.0, 20.0, 10.0] and note == "no net power lost, nothing to share by inertia"
    with pytest.raises(ValueError):
        share_lost_power(m, units, m.bus_type, math.nan, "droop")
    with pytest.raises(ValueError):
        share_lost_power(m, units, m.bus_type, 5.0, "reference")
    # a crossed Pmin / Pmax is refused only on a unit that takes part (ParticipationWeights, :1634-1641)
    crossed = converters_model()
    crossed.pmin[1], crossed.pmax[1] = 300.0, 200.0   # the wind plant: a converter, so it takes no part
    pg, _ = share_lost_power(crossed, units, crossed.bus_type, 10.0, "droop")
    assert pg[0] == 40.0
    crossed.pmin[0] = 60.0                            # the synchronous unit: refused
    with pytest.raises(ValueError, match="Pmin 60 MW above Pmax 50 MW"):
        share_lost_power(crossed, units, crossed.bus_type, 10.0, "droop")


def test_shared_rows_are_merged_in_outage_order():
    from gridsim_b200.engine import _merge_rows
    raw = dict(status=np.array([0, 0, 1], np.int32), iterations=np.array([3, 4, 20], np.int32),
               max_mismatch=np.zeros(3), min_vm=np.array([0.97, 0.98, 0.0]), max_vm=np.array([1.02, 1.03, 0.0]),
               max_loading_pct=np.array([90.0, 101.0, 0.0]), worst_boundary_pct=np.zeros(3),
               islanded=np.zeros(3, np.uint8), viol_ptr=np.array([0, 0, 1, 1], np.int32),
               viol_kind=np.array([0], np.int32), viol_element=np.array([7], np.int32), viol_value=np.array([101.0]))
    sub = dict(status=np.array([0], np.int32), iterations=np.array([5], np.int32), max_mismatch=np.zeros(1),
               min_vm=np.array([0.93]), max_vm=np.array([1.01]), max_loading_pct=np.array([120.0]),
               worst_boundary_pct=np.zeros(1), islanded=np.zeros(1, np.uint8), viol_ptr=np.array([0, 2], np.int32),
               viol_kind=np.array([0, 2], np.int32), viol_element=np.array([4, 11], np.int32),
               viol_value=np.array([120.0, 0.93]))
    _merge_rows(raw, {0: sub}, keep_states=False)
    assert list(raw["status"]) == [0, 0, 1] and list(raw["iterations"]) == [5, 4, 20]
    assert list(raw["viol_ptr"]) == [0, 2, 3, 3]
    assert list(raw["viol_kind"]) == [0, 2, 0] and list(raw["viol_element"]) == [4, 11, 7]
    assert list(raw["viol_value"]) == [120.0, 0.93, 101.0] and raw["viol_kind"].dtype == np.int32


def test_bad_dispatch_options_are_refused_before_any_device_call():
    """An unknown dispatch, and a warm start with a shared one, fail before the library is reached (no device here)."""
    m = n124()
    solver = SparseNewtonRaphsonPowerFlow()
    with pytest.raises(ValueError, match="unknown outage dispatch"):
        ContingencyAnalysis.screen_elements_raw(m, [1], [0], solver, PowerFlowOptions(), dispatch="proportional")
    with pytest.raises(ValueError, match="warm_start_from_base"):
        ContingencyAnalysis.screen_elements_raw(m, [1], [0], solver, PowerFlowOptions(warm_start_from_base=True),
                                                dispatch="droop")
