"""The screen's topology pass on the host (no GPU): which outages split the network (ContingencyAnalysis.Splits,
Analysis/ContingencyAnalysis.cs:1665-1687) and which leave a part ProvablyUnsolvablePart (:1750-1830) rejects.

The engine's pass (``gs_outage_topology``: one depth-first search, bridges and preorder sums) is checked outage by
outage against the oracle, which rebuilds the reduced model and runs the reference's union-find per outage; and
against the cases the reference's own tests pin (Lf2ContainedTests.N232.cs, ContingencyIslandedLabelTests.cs).
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import synthetic
from gridsim_b200.engine import ContingencyAnalysis
from gridsim_b200.model import PQ, PV, SLACK, GridModel
from tests.conftest import golden_model

TOL = 1e-8


def _both(m, idx, tol=TOL):
    got = ContingencyAnalysis.outage_topology(m, idx, tol)
    ref = oracle.outage_topology(m, idx, tol)
    return got, ref


def _bid(m, f, t):
    pos = {int(b): i for i, b in enumerate(m.bus_id)}
    ks = [k for k in range(m.n_branch) if m.br_from[k] == pos[f] and m.br_to[k] == pos[t]]
    assert len(ks) == 1
    return ks[0]


@pytest.mark.parametrize("name", ["case9", "case14", "case57", "case118", "case300"])
def test_every_branch_outage_matches_the_oracle(name):
    m, _ = golden_model(name)
    idx = np.concatenate([[-1], np.arange(m.n_branch)]).astype(np.int32)
    (sp, un), (rsp, run) = _both(m, idx)
    assert np.array_equal(sp, rsp)
    assert np.array_equal(un, run)
    assert not un[0]  # a connected model has no unsolvable part (N232_a_connected_model_has_no_unsolvable_part)


def test_case9_islanded_outages_take_the_shortcut():
    # N232_the_documented_case9_islanded_outages_take_the_shortcut_and_keep_their_verdict: 1-4 (buses 2-9 lose the
    # reference: 248 MW of units against 315 MW of demand), 3-6 and 8-2 (a generator bus alone, lossless).
    m, _ = golden_model("case9")
    idx = np.array([_bid(m, 1, 4), _bid(m, 3, 6), _bid(m, 8, 2), _bid(m, 4, 5)], np.int32)
    sp, un = ContingencyAnalysis.outage_topology(m, idx)
    assert sp.tolist() == [True, True, True, False]
    assert un.tolist() == [True, True, True, False]


def test_case14_condenser_cut_off_is_still_solved():
    # N232_the_case14_condenser_cut_off_by_7_8_is_still_solved: bus 8 (Pg = 0, no load, no shunt) is cut off, but
    # its P equation holds, so no proof applies.
    m, _ = golden_model("case14")
    sp, un = ContingencyAnalysis.outage_topology(m, [_bid(m, 7, 8)])
    assert sp[0] and not un[0]


def _three_bus(pg2, pd3, r23, gs3=0.0, type2=PV):
    """N232ThreeBus: bus 1 the reference with a unit, {2, 3} a part with no reference (the 1-2 branch is out)."""
    return GridModel(
        name="three", base_mva=100.0, bus_id=np.array([1, 2, 3], np.int32),
        bus_type=np.array([SLACK, type2, PQ], np.int32), pd=np.array([0.0, 0.0, pd3]), qd=np.zeros(3),
        gs=np.array([0.0, 0.0, gs3]), bs=np.zeros(3), vm=np.ones(3), va_deg=np.zeros(3), vmin=np.full(3, np.nan),
        vmax=np.full(3, np.nan), base_kv=np.full(3, 100.0), gen_bus=np.array([0, 1], np.int32),
        pg=np.array([50.0, pg2]), qg=np.zeros(2), vg=np.ones(2), qmin=np.full(2, -100.0), qmax=np.full(2, 100.0),
        gen_in_service=np.ones(2, np.uint8), br_from=np.array([0, 1], np.int32), br_to=np.array([1, 2], np.int32),
        r=np.array([0.01, r23]), x=np.array([0.1, 0.1]), b=np.zeros(2), tap=np.ones(2), shift_deg=np.zeros(2),
        rate_a=np.zeros(2), br_in_service=np.array([0, 1], np.uint8), is_transformer=np.zeros(2, np.uint8))


@pytest.mark.parametrize("pg2,pd3,r23,gs3,expect", [
    (10, 30, 0.01, 0.0, True),    # load part (demand > units, R >= 0)
    (30, 10, 0.0, 0.0, True),     # lossless, surplus
    (10, 30, 0.0, 0.0, True),     # lossless, deficit
    (30, 10, 0.01, 0.0, False),   # lossy with a surplus: the losses might absorb it
    (10, 10, 0.0, 0.0, False),    # balanced within the margin
    (10, 30, 0.01, -1.0, False),  # a negative shunt conductance: no proof
])
def test_the_proof_covers_only_what_it_proves(pg2, pd3, r23, gs3, expect):
    # N232_the_proof_covers_only_what_it_proves, on the intact model (-1) and on the outage of the 2-3 branch
    m = _three_bus(pg2, pd3, r23, gs3)
    (sp, un), (rsp, run) = _both(m, [-1, 1])
    assert un[0] == expect
    assert np.array_equal(sp, rsp) and np.array_equal(un, run)
    # out-of-service branch 0 joins nothing, so the outage of 2-3 splits {2, 3}
    assert sp.tolist() == [False, True]


def _random_grid(seed):
    """A small random network: a spanning tree plus a few chords (parallel branches among them), random losses
    (some zero, the odd negative), units and loads, sometimes a second part cut off by an out-of-service branch."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(4, 26))
    f, t = [], []
    for i in range(1, n):
        f.append(int(rng.integers(0, i)))
        t.append(i)
    for _ in range(int(rng.integers(0, n // 2 + 1))):
        a, b = rng.choice(n, 2, replace=False)
        f.append(int(a))
        t.append(int(b))
    if rng.random() < 0.3 and len(f) > 2:  # a parallel branch
        f.append(f[0])
        t.append(t[0])
    nb = len(f)
    on = np.ones(nb, np.uint8)
    if rng.random() < 0.3:
        on[int(rng.integers(0, n - 1))] = 0  # a tree branch out of service: possibly a second part
    r = np.where(rng.random(nb) < 0.4, 0.0, rng.uniform(0.001, 0.05, nb))
    if rng.random() < 0.1:
        r[int(rng.integers(0, nb))] = -0.001
    gs = np.where(rng.random(n) < 0.8, 0.0, rng.uniform(0.0, 2.0, n))
    btype = np.full(n, PQ, np.int32)
    btype[0] = SLACK
    ng = int(rng.integers(1, max(2, n // 3)))
    gbus = np.concatenate([[0], rng.choice(np.arange(1, n), ng - 1, replace=False)]).astype(np.int32) if ng > 1 \
        else np.array([0], np.int32)
    btype[gbus[1:]] = PV
    pg = np.round(rng.uniform(0, 80, gbus.shape[0]), 1)
    pd = np.where(rng.random(n) < 0.5, 0.0, np.round(rng.uniform(0, 60, n), 1))
    if rng.random() < 0.3:
        pd[int(rng.integers(0, n))] = 0.0
    return GridModel(
        name=f"rand{seed}", base_mva=100.0, bus_id=np.arange(1, n + 1, dtype=np.int32), bus_type=btype, pd=pd,
        qd=np.zeros(n), gs=gs, bs=np.zeros(n), vm=np.ones(n), va_deg=np.zeros(n), vmin=np.full(n, np.nan),
        vmax=np.full(n, np.nan), base_kv=np.full(n, 100.0), gen_bus=gbus, pg=pg, qg=np.zeros(gbus.shape[0]),
        vg=np.ones(gbus.shape[0]), qmin=np.full(gbus.shape[0], -99.0), qmax=np.full(gbus.shape[0], 99.0),
        gen_in_service=np.ones(gbus.shape[0], np.uint8), br_from=np.array(f, np.int32), br_to=np.array(t, np.int32),
        r=r, x=np.full(nb, 0.1), b=np.zeros(nb), tap=np.ones(nb), shift_deg=np.zeros(nb), rate_a=np.zeros(nb),
        br_in_service=on, is_transformer=np.zeros(nb, np.uint8))


def test_random_networks_match_the_oracle():
    seen_split = seen_unsolvable = 0
    for seed in range(300):
        m = _random_grid(seed)
        idx = np.arange(-1, m.n_branch, dtype=np.int32)
        (sp, un), (rsp, run) = _both(m, idx)
        assert np.array_equal(sp, rsp), seed
        assert np.array_equal(un, run), seed
        seen_split += int(sp.sum())
        seen_unsolvable += int(un.sum())
    assert seen_split > 100 and seen_unsolvable > 50  # the sample exercises both verdicts


def test_synthetic_grids_match_the_oracle():
    for cfg in (0, 1):
        m = synthetic.config_grid(cfg, 0)
        idx = np.arange(-1, m.n_branch, dtype=np.int32)
        (sp, un), (rsp, run) = _both(m, idx)
        assert np.array_equal(sp, rsp) and np.array_equal(un, run)
