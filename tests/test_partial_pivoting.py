"""Row partial pivoting on the device, against the oracle (the reference's FP64 Gilbert-Peierls factorisation with
row partial pivoting, SparseLuFactorization.cs:69-195).

* The batched sparse solve (gs_sparse_solve_batch, ISparseLinearSolver / IBatchedSparseLinearSolver): matrices whose
  stored diagonal is zero collapse every static diagonal pivot; they are solved again with row partial pivoting and
  match dense solves and the oracle. A singular matrix is still reported singular.
* The Newton solve: a grid built so that a static pivot collapses at the start (a resistive leaf,
  conftest.resistive_leaf_grid; the CPU test in test_host_logic.py shows the collapse under the oracle's order) is
  re-solved with partial pivoting and equals the oracle, in both precisions, through single solves and a screen
  whose every outage starts at the collapsing point (n_partial_pivot counts them, n_singular_pivot stays 0).
* The `partial_pivoting` option (every step of every system by that factorisation) on the golden cases and a case118
  screen: identical statuses, iteration counts and violation lists, states within 1e-8.
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import (ContingencyAnalysis, CudaSparseLinearSolver, PowerFlowOptions,
                                 SparseNewtonRaphsonPowerFlow)
from tests.conftest import golden_model, resistive_leaf_grid

pytestmark = pytest.mark.gpu

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8


def _csr(a):
    rows, cols = np.nonzero(np.ones_like(a, bool) & ((a != 0) | np.eye(a.shape[0], dtype=bool)))
    indptr = np.searchsorted(rows, np.arange(a.shape[0] + 1)).astype(np.int32)
    return indptr, cols.astype(np.int32), a[rows, cols].astype(np.float64)


def _zero_diagonal_matrix(n, seed):
    """A regular matrix whose diagonal is stored but zero: a row permutation (no fixed point) of a diagonally
    dominant sparse matrix, with the diagonal cells present."""
    rng = np.random.default_rng(seed)
    a = np.zeros((n, n))
    for i in range(n):
        for j in rng.choice(n, 3, replace=False):
            a[i, j] = rng.uniform(-1, 1)
        a[i, i] = 4.0 + rng.uniform(0, 1)
    perm = np.roll(np.arange(n), 1 + seed % (n - 1))
    p = a[perm]
    np.fill_diagonal(p, 0.0)
    p[np.arange(n), perm] = a[perm, perm]  # keep the dominant entries where the permutation put them
    return p


def test_sparse_solve_pivots_off_a_zero_diagonal():
    solver = CudaSparseLinearSolver()
    mats, rhs = [], []
    small = np.array([[0.0, 2.0, 1.0], [2.0, 0.0, 3.0], [1.0, 3.0, 0.0]])
    mats.append(small)
    for k, n in enumerate((8, 40, 200)):
        mats.append(_zero_diagonal_matrix(n, k + 1))
    rng = np.random.default_rng(0)
    rhs = [rng.uniform(-1, 1, a.shape[0]) for a in mats]
    got = solver.solve_batch([_csr(a) for a in mats], rhs)
    for a, b, x in zip(mats, rhs, got):
        assert x is not None
        ref = np.linalg.solve(a, b)
        assert np.max(np.abs(x - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))
        rp, ci, val = _csr(a)
        xo = oracle.sparse_solve(rp, ci, val, b)
        assert xo is not None and np.max(np.abs(x - xo)) <= 1e-12 * max(1.0, np.max(np.abs(xo)))
    # a singular matrix (third row the sum of the others) whose first diagonal entry is zero stays singular
    sing = np.array([[0.0, 1.0, 2.0], [1.0, 0.0, 1.0], [1.0, 1.0, 3.0]])
    assert oracle.sparse_solve(*_csr(sing), np.ones(3)) is None
    assert solver.solve_batch([_csr(sing)], [np.ones(3)]) == [None]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_collapsing_static_pivot_is_resolved_with_partial_pivoting(precision):
    m = resistive_leaf_grid()
    opt = PowerFlowOptions(max_iterations=20, precision=precision)
    ref = oracle.solve(m, opt.to_c())
    assert ref["status"] == _abi.PF_CONVERGED
    got = SparseNewtonRaphsonPowerFlow(precision).solve(m, opt)
    assert got.status == ref["status"] and got.iterations == ref["iterations"]
    assert np.max(np.abs(got.vm - ref["vm"])) <= VM_TOL
    assert np.max(np.abs(np.radians(got.va_deg - ref["va_deg"]))) <= VA_TOL_RAD
    # a screen without the warm start: every outage starts at the collapsing point
    bridge = synthetic.bridges(m)
    idx = np.array([k for k in range(m.n_branch) if not bridge[k]], np.int32)
    sopt = PowerFlowOptions(max_iterations=20, precision=precision, per_bus_voltage_limits=True)
    g = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow(precision), sopt, keep_states=True)
    r = oracle.screen(m, idx, sopt.to_c(), keep_states=True)
    assert g["n_singular_pivot"] == 0
    solved = np.sum(r["status"] != _abi.PF_UNSOLVABLE_PART)
    assert g["n_partial_pivot"] == solved > 0
    assert np.array_equal(g["status"], r["status"])
    assert np.array_equal(g["iterations"], r["iterations"])
    conv = r["status"] == _abi.PF_CONVERGED
    assert np.max(np.abs(g["vm"][conv] - r["vm"][conv])) <= VM_TOL
    assert np.max(np.abs(np.radians(g["va_deg"][conv] - r["va_deg"][conv]))) <= VA_TOL_RAD
    assert np.array_equal(g["viol_ptr"], r["viol_ptr"]) and np.array_equal(g["viol_element"], r["viol_element"])


@pytest.mark.parametrize("case", ["case9", "case57", "case118", "case300"])
def test_partial_pivoting_option_matches_the_oracle(case):
    m, _ = golden_model(case)
    opt = PowerFlowOptions(max_iterations=20, partial_pivoting=True)
    ref = oracle.solve(m, PowerFlowOptions(max_iterations=20).to_c())
    got = SparseNewtonRaphsonPowerFlow("fp64").solve(m, opt)
    assert got.status == ref["status"] and got.iterations == ref["iterations"]
    if ref["status"] == _abi.PF_CONVERGED:
        assert np.max(np.abs(got.vm - ref["vm"])) <= VM_TOL
        assert np.max(np.abs(np.radians(got.va_deg - ref["va_deg"]))) <= VA_TOL_RAD


def test_partial_pivoting_screen_of_case118_matches_the_oracle():
    m, _ = golden_model("case118")
    idx = np.asarray(m.in_service_branches(), np.int32)
    opt = PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True, warm_start_from_base=True,
                           partial_pivoting=True)
    g = ContingencyAnalysis.screen_raw(m, idx, SparseNewtonRaphsonPowerFlow("fp64"), opt, keep_states=True)
    r = oracle.screen(m, idx, opt.to_c(), keep_states=True)
    assert np.array_equal(g["status"], r["status"])
    assert np.array_equal(g["iterations"], r["iterations"])
    conv = r["status"] == _abi.PF_CONVERGED
    assert np.max(np.abs(g["vm"][conv] - r["vm"][conv])) <= VM_TOL
    assert np.max(np.abs(np.radians(g["va_deg"][conv] - r["va_deg"][conv]))) <= VA_TOL_RAD
    assert np.array_equal(g["viol_ptr"], r["viol_ptr"])
    assert np.array_equal(g["viol_kind"], r["viol_kind"]) and np.array_equal(g["viol_element"], r["viol_element"])
