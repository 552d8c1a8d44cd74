"""The oracle pinned against the reference's own known answers (CPU only).

Sources: PowerFlowTests.cs:11-15,38-60 (case9), IeeeCasesTests.cs:16-24,91-95 (case14/57/118/300),
ContingencyCorrectnessTests.cs:143-154 (case118 N-1 counts), :209-237 (case14 base case and raw counts).
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi
from tests.conftest import golden_model


@pytest.mark.parametrize("name", ["case9", "case14", "case57", "case118", "case300"])
def test_published_voltages(name):
    m, pub = golden_model(name)
    o = _abi.default_opts()
    o.enforce_q_limits = 1  # the reference tests solve with the default options (Q limits on)
    r = oracle.solve(m, o)
    assert r["status"] == _abi.PF_CONVERGED
    assert r["max_mismatch"] < 1e-8
    slack = int(np.nonzero(m.bus_type == 3)[0][0])
    va = r["va_deg"] - r["va_deg"][slack] + pub["va_deg"][slack]  # re-referenced as IeeeCasesTests does
    assert np.max(np.abs(r["vm"] - pub["vm"])) <= pub["vm_tol"]
    assert np.max(np.abs(va - pub["va_deg"])) <= pub["va_tol_deg"]


def test_case9_slack_and_losses():
    m, _ = golden_model("case9")
    r = oracle.solve(m)
    assert abs(r["p_inj_mw"][0] - 71.64) < 0.05   # PowerFlowTests.cs:52-55
    assert abs(r["p_inj_mw"].sum() - 4.641) < 0.005
    assert r["iterations"] <= 6


def test_case9_iteration_cap_reports_max_iterations():
    m, _ = golden_model("case9")
    o = _abi.default_opts()
    o.max_iterations = 1
    o.flat_start = 1
    r = oracle.solve(m, o)
    assert r["status"] == _abi.PF_MAX_ITERATIONS  # PowerFlowTests.cs:27-36


def _counts(r):
    conv = r["status"] == _abi.PF_CONVERGED
    nv = np.diff(r["viol_ptr"])
    return int(np.sum(conv & (nv == 0))), int(np.sum(conv & (nv > 0))), int(np.sum(~conv))


def test_case118_n1_counts_under_study_options(study_opts):
    m, _ = golden_model("case118")
    r = oracle.screen(m, m.in_service_branches(), study_opts)
    assert _counts(r) == (164, 13, 9)


def test_case14_base_and_raw_counts(study_opts):
    m, _ = golden_model("case14")
    b = oracle.screen(m, np.zeros(0, np.int32), study_opts)
    # the base case through the same classification: solve the intact grid as a screen of no outage
    base = oracle.solve(m, study_opts)
    assert base["status"] == _abi.PF_CONVERGED
    over = [int(m.bus_id[i]) for i in range(m.n_bus) if base["vm"][i] > 1.06]
    assert over == [6, 7, 8]
    assert abs(base["vm"][list(m.bus_id).index(8)] - 1.09) < 1e-12
    raw = oracle.screen(m, m.in_service_branches(), study_opts)
    assert _counts(raw) == (0, 19, 1)
    assert b["viol_ptr"].shape == (1,)


def test_max_mismatch_of_screen_states_is_the_screens_own():
    """oracle.max_mismatch (the checker of the allocation-free entry point) gives, for the states an N-1 screen
    ends in, the max mismatch that screen reports for them (both cut short after two steps, so they are large)."""
    from gridsim_b200 import synthetic
    m = synthetic.config_grid(0, 0)
    idx = synthetic.outage_set(m, None, 0)[:24].astype(np.int32)
    o = _abi.default_opts()
    o.max_iterations = 2
    o.warm_start_from_base = 0
    r = oracle.screen(m, idx, o, keep_states=True)
    got = oracle.max_mismatch(m, r["vm"], np.radians(r["va_deg"]), idx)
    assert np.allclose(got, r["max_mismatch"], rtol=1e-9, atol=1e-13)
    assert got.max() > 1e-6
    intact = oracle.max_mismatch(m, r["vm"], np.radians(r["va_deg"]))
    assert not np.allclose(intact, got)


def _dense_csr(a):
    """CSR of a dense matrix: its nonzero cells and the diagonal."""
    a = np.asarray(a, float)
    rp, ci, v = [0], [], []
    for i, row in enumerate(a):
        for j, x in enumerate(row):
            if x != 0.0 or i == j:
                ci.append(j)
                v.append(x)
        rp.append(len(ci))
    return rp, ci, v


def test_ilu0_guard_is_relative_at_a_tiny_scale():
    """NumericTolerancesTests.cs:287-301 (Ilu0_guard_is_relative_so_a_small_scale_matrix_keeps_its_exact_factors):
    for a 2 x 2 matrix ILU(0) is the full LU, so Apply solves A z = r exactly even at scale 1e-14."""
    s = 1e-14
    z = oracle.ilu0_apply(*_dense_csr([[4 * s, 1 * s], [1 * s, 3 * s]]), [5 * s, 4 * s])
    assert abs(z[0] - 1.0) < 1e-12 and abs(z[1] - 1.0) < 1e-12


def test_ilu0_guard_regularises_a_zero_pivot():
    """NumericTolerancesTests.cs:303-310: a structurally zero second pivot is pushed to 1e-12 x its row scale, so
    Apply stays finite."""
    z = oracle.ilu0_apply(*_dense_csr([[1, 1], [1, 1]]), [1.0, 1.0])
    assert np.all(np.isfinite(z))


def test_bicgstab_solves_the_reference_two_by_two():
    """NumericTolerancesTests.cs:312-323: BiCGSTAB with the default tolerance and cap solves [[4,1],[1,3]] x = [5,4]
    to x = [1, 1] (ten decimals)."""
    ok, x = oracle.bicgstab(*_dense_csr([[4, 1], [1, 3]]), [5.0, 4.0])
    assert ok
    assert x == pytest.approx([1.0, 1.0], abs=5e-11)


def test_bicgstab_on_a_larger_system_matches_a_dense_solve():
    """The same pieces on a sparse, diagonally dominant 200 x 200 system: accepted, and within the true-residual
    tolerance of the dense solution."""
    rng = np.random.default_rng(5)
    n = 200
    a = np.zeros((n, n))
    for i in range(n):
        for j in rng.choice(n, 4, replace=False):
            a[i, j] = rng.uniform(-1, 1)
        a[i, i] = np.sum(np.abs(a[i])) + 1.0
    b = rng.uniform(-1, 1, n)
    ok, x = oracle.bicgstab(*_dense_csr(a), b)
    assert ok
    want = np.linalg.solve(a, b)
    assert np.linalg.norm(a @ x - b) / np.linalg.norm(b) < 1e-10
    assert np.max(np.abs(x - want)) < 1e-8
