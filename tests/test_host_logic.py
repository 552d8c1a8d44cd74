"""Host-side logic on CPU: netting against the base case, violation texts, option mapping, sharding."""
import numpy as np

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import ContingencyAnalysis, PowerFlowOptions
from gridsim_b200.parallel import balanced_shards, merge, outage_costs, reorder, shard
from tests.conftest import golden_model


def _study():
    o = _abi.default_opts()
    o.max_iterations = 100
    o.enforce_q_limits = 1
    return o


def test_case14_netting_pins():
    """ContingencyCorrectnessTests.cs:209-237: base overvoltage 1.090 on buses 6, 7, 8; netted 16 / 3 / 1."""
    m, _ = golden_model("case14")
    o = _study()
    base = ContingencyAnalysis._results(m, [-1], oracle.screen(m, np.array([-1], np.int32), o))[0]
    assert base.violations == ["overvoltage 1.090 p.u."]
    assert [d.element for d in base.details] == [6, 7, 8]
    assert abs(base.details[0].value - 1.07) < 1e-12
    idx = m.in_service_branches()
    raw = ContingencyAnalysis._results(m, idx, oracle.screen(m, idx, o))
    net = [ContingencyAnalysis.net_against_base(m, r, base) for r in raw]
    assert sum(r.secure for r in net) == 16
    assert sum(r.converged and not r.secure for r in net) == 3
    assert sum(not r.converged for r in net) == 1
    for r in net:
        if r.converged:
            assert "overvoltage 1.090 p.u." in r.pre_existing_violations


def test_violation_texts_follow_the_reference_format():
    from gridsim_b200.engine import ContingencyViolation, _violation_texts
    m, _ = golden_model("case14")
    det = [ContingencyViolation(_abi.VIOL_BRANCH_OVERLOAD, 0, 104.4, "1-2"),
           ContingencyViolation(_abi.VIOL_UNDERVOLTAGE, 5, 0.93412, ""),
           ContingencyViolation(_abi.VIOL_UNDERVOLTAGE, 6, 0.9312, ""),
           ContingencyViolation(_abi.VIOL_OVERVOLTAGE, 8, 1.0901, "")]
    assert _violation_texts(m, det) == ["branch 1-2 104%", "undervoltage 0.931 p.u.", "overvoltage 1.090 p.u."]


def test_options_map_onto_the_c_struct():
    c = PowerFlowOptions(tolerance=1e-9, max_iterations=7, precision="mixed", warm_start_from_base=True,
                         per_bus_voltage_limits=True, batch_width=64).to_c()
    assert (c.tolerance, c.max_iterations, c.precision, c.warm_start_from_base, c.per_bus_voltage_limits,
            c.batch_width) == (1e-9, 7, _abi.PREC_MIXED, 1, 1, 64)


def test_shards_cover_every_outage_once():
    for n in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            covered = []
            for r in range(world):
                covered.extend(range(n)[shard(n, r, world)])
            assert covered == list(range(n))


def test_merged_shards_equal_one_screen():
    m = synthetic.config_grid(0, 0)
    idx = synthetic.outage_set(m, None, 0)[:30]
    o = _abi.default_opts()
    o.max_iterations = 20
    o.per_bus_voltage_limits = 1
    o.warm_start_from_base = 1
    whole = oracle.screen(m, idx, o)
    parts = [oracle.screen(m, idx[shard(len(idx), r, 3)], o) for r in range(3)]
    got = merge(parts)
    for k in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element"):
        assert np.array_equal(got[k], whole[k]), k
    assert np.array_equal(got["viol_value"], whole["viol_value"])


def test_balanced_shards_cover_every_row_once_and_even_the_costs():
    rng = np.random.default_rng(3)
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            costs = rng.uniform(2.3, 20.0, n)
            shards = balanced_shards(costs, world)
            assert sorted(np.concatenate(shards).tolist()) == list(range(n))
            assert all(np.all(np.diff(s) > 0) for s in shards)
            if n >= world:
                sums = [costs[s].sum() for s in shards]
                # longest processing time first: no rank exceeds the others by more than the largest single cost
                assert max(sums) - min(sums) <= costs.max() + 1e-9
    # equal costs: counts differ by at most one
    shards = balanced_shards(np.ones(101), 8)
    assert max(len(s) for s in shards) - min(len(s) for s in shards) <= 1


def test_outage_costs_follow_the_removed_flow():
    m = synthetic.config_grid(1, 0)
    idx = synthetic.outage_set(m, None, 0)[:200]
    c = outage_costs(m, idx)
    assert c.shape == (200,) and np.all(c >= 2.3) and np.all(c <= 20.0)
    th = np.radians(m.va_deg)
    flow = np.abs(th[m.br_from[idx]] - th[m.br_to[idx]] - np.radians(m.shift_deg[idx])) / np.abs(m.x[idx])
    assert np.array_equal(np.argsort(c, kind="stable"), np.argsort(flow, kind="stable"))
    sets = np.stack([idx[:50], np.where(np.arange(50) % 2 == 0, idx[50:100], -1)], axis=1)
    cs = outage_costs(m, sets, "sets")
    assert np.all(cs >= c[:50] - 1e-12)
    on = np.nonzero(m.gen_in_service)[0][:5]
    rows = np.array([[0, int(idx[0])]] + [[1, int(g)] for g in on] + [[2, 3]], np.int32)
    ce = outage_costs(m, rows, "elements")
    assert ce[0] == c[0] and ce.shape == (7,)


def test_reordered_balanced_merge_equals_one_screen():
    m = synthetic.config_grid(0, 0)
    idx = synthetic.outage_set(m, None, 0)[:40]
    o = _abi.default_opts()
    o.max_iterations = 20
    o.per_bus_voltage_limits = 1
    o.warm_start_from_base = 1
    whole = oracle.screen(m, idx, o)
    shards = balanced_shards(outage_costs(m, idx), 3)
    parts = [oracle.screen(m, idx[s], o) for s in shards]
    got = reorder(merge(parts), np.concatenate(shards))
    for k in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "max_loading_pct"):
        assert np.array_equal(got[k], whole[k]), k
    assert np.array_equal(got["viol_value"], whole["viol_value"])


def test_resistive_leaf_collapses_a_static_diagonal_pivot():
    """The crafted grid of the partial-pivoting GPU tests: under the oracle's minimum-degree order the static
    diagonal elimination of its start Jacobian meets a zero pivot, the matrix is regular, and the oracle (row partial
    pivoting) converges."""
    from tests.conftest import resistive_leaf_grid
    m = resistive_leaf_grid()
    rp, ci, val, _ = oracle.jacobian(m)
    n = len(rp) - 1
    a = np.zeros((n, n))
    for i in range(n):
        a[i, ci[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    q = oracle.md_order(rp, ci)
    p = a[np.ix_(q, q)].copy()
    collapsed = False
    for k in range(n):
        if abs(p[k, k]) <= 1e-12 * max(1.0, abs(p[k, k])):
            collapsed = True
            break
        p[k + 1:, k] /= p[k, k]
        p[k + 1:, k + 1:] -= np.outer(p[k + 1:, k], p[k, k + 1:])
    assert collapsed
    assert np.linalg.cond(a) < 1e4
    o = _abi.default_opts()
    o.max_iterations = 20
    assert oracle.solve(m, o)["status"] == _abi.PF_CONVERGED
