"""The seeded synthetic grids of the benchmark workloads (CPU)."""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.model import load_case_dir, save_case_dir


def test_sizes_and_determinism():
    a = synthetic.config_grid(0, 3)
    b = synthetic.config_grid(0, 3)
    assert (a.n_bus, a.n_branch, int(np.sum(a.bus_type == 2)), int(np.sum(a.bus_type == 3))) == (120, 180, 20, 1)
    for k, v in a.__dict__.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, getattr(b, k), equal_nan=True), k
    assert int(np.sum(a.is_transformer)) == 18
    assert np.all(a.rate_a >= 1.0)


def test_stored_start_is_a_solution():
    m = synthetic.config_grid(1, 0)
    r = oracle.solve(m)
    assert r["status"] == _abi.PF_CONVERGED
    assert r["iterations"] <= 1
    assert m.meta["load_scale"] > 0


def test_bridges_match_brute_force():
    m = synthetic.make_grid(40, 50, 6, 11, operating_point=False)
    br = synthetic.bridges(m)
    for k in range(m.n_branch):
        keep = np.ones(m.n_branch, bool)
        keep[k] = False
        parent = list(range(m.n_bus))

        def find(x):
            while parent[x] != x:
                parent[x] = parent[parent[x]]
                x = parent[x]
            return x
        for j in np.nonzero(keep)[0]:
            ra, rb = find(int(m.br_from[j])), find(int(m.br_to[j]))
            if ra != rb:
                parent[ra] = rb
        parts = len({find(i) for i in range(m.n_bus)})
        assert br[k] == (parts > 1), k


def test_outage_sets_avoid_islanding():
    m = synthetic.config_grid(0, 0)
    idx = synthetic.outage_set(m, None, 0)
    assert not np.any(synthetic.bridges(m)[idx])
    sub = synthetic.outage_set(m, 50, 0)
    assert len(sub) == 50 and np.all(np.isin(sub, idx))


def test_case_directory_round_trip(tmp_path):
    m = synthetic.config_grid(0, 0)
    save_case_dir(m, str(tmp_path / "case"))
    back = load_case_dir(str(tmp_path / "case"))
    assert back.n_bus == m.n_bus and back.n_branch == m.n_branch
    for k in ("pd", "qd", "vm", "va_deg", "r", "x", "b", "tap", "rate_a", "pg", "vg"):
        assert np.allclose(getattr(back, k), getattr(m, k), rtol=0, atol=1e-12), k
    assert np.array_equal(back.bus_type, m.bus_type)
    r1, r2 = oracle.solve(m), oracle.solve(back)
    assert np.allclose(r1["vm"], r2["vm"], atol=1e-12)


def test_stressed_operating_point_is_a_solution_closer_to_the_limit():
    """margin 0.9 (the stressed screen): the stored start still solves, at 1.5 x the load of the default 0.6 margin
    (both a fraction of the same last solvable level), and its outages take at least as many Newton steps."""
    base = synthetic.config_grid(1, 0)
    stressed = synthetic.config_grid(1, 0, margin=0.9)
    r = oracle.solve(stressed)
    assert r["status"] == _abi.PF_CONVERGED
    assert r["iterations"] <= 1
    assert stressed.meta["load_scale"] / base.meta["load_scale"] == pytest.approx(0.9 / 0.6, rel=1e-12)
    assert np.array_equal(stressed.tap, base.tap) and np.array_equal(stressed.vg, base.vg)
    idx = np.arange(0, 40, dtype=np.int32)
    it_base = oracle.screen(base, idx)["iterations"]
    it_stressed = oracle.screen(stressed, idx)["iterations"]
    assert np.sum(it_stressed) >= np.sum(it_base)
