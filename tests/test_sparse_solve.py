"""The batched sparse linear solve (gs_sparse_solve_batch: ISparseLinearSolver.Solve and
IBatchedSparseLinearSolver.SolveBatch, Abstractions/ISparseLinearSolver.cs:12-17, IBatchedSparseLinearSolver.cs:19-37).

CPU: the oracle's restatement of the reference's solver (CpuSparseLuSolver over the Gilbert-Peierls LU with partial
pivoting) against dense numpy solves, which pins it on arbitrary matrices. GPU: systems of different sizes and
patterns in one call (the reference's Jacobians of the golden cases at their start points, random nonsymmetric
diagonally dominant matrices) against the oracle, within REL_TOL of the solution's norm (FP64 with a different
pivot order: the results agree to rounding); singular systems give no result, non-finite and malformed systems an
error for that system alone, and the inputs are left as they were.
"""
import numpy as np
import pytest

import oracle
from gridsim_b200 import synthetic
from tests.conftest import golden_model

REL_TOL = 1e-9


def _random_csr(n, seed, density=0.08):
    rng = np.random.default_rng(seed)
    a = np.where(rng.random((n, n)) < density, rng.normal(size=(n, n)), 0.0)
    a += np.diag(np.abs(a).sum(axis=1) + 1.0 + rng.random(n))  # diagonally dominant: the diagonal pivots hold
    rows, cols = np.nonzero(a)
    indptr = np.searchsorted(rows, np.arange(n + 1)).astype(np.int32)
    return (indptr, cols.astype(np.int32), a[rows, cols]), a


def test_oracle_solver_matches_dense_solves():
    for seed in range(20):
        (rp, ci, v), a = _random_csr(int(5 + 7 * seed), seed)
        b = np.random.default_rng(seed + 99).normal(size=a.shape[0])
        x = oracle.sparse_solve(rp, ci, v, b)
        ref = np.linalg.solve(a, b)
        assert np.max(np.abs(x - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_oracle_solver_reports_singular():
    (rp, ci, v), a = _random_csr(12, 3)
    v = v.copy()
    v[rp[4]:rp[5]] = 0.0  # a zero row
    assert oracle.sparse_solve(rp, ci, v, np.ones(12)) is None


def _jacobians():
    out = []
    for name in ("case9", "case14", "case57", "case118", "case300"):
        m, _ = golden_model(name)
        rp, ci, v, mis = oracle.jacobian(m)
        out.append(((rp, ci, v), mis))
    m = synthetic.config_grid(1, 0)
    rp, ci, v, mis = oracle.jacobian(m)
    out.append(((rp, ci, v), mis))
    return out


@pytest.mark.gpu
def test_mixed_batch_matches_the_oracle():
    from gridsim_b200.engine import CudaSparseLinearSolver
    systems = []
    for (csr, mis) in _jacobians():
        rng = np.random.default_rng(len(systems))
        for c in range(3):  # the same pattern three times, values perturbed
            v = csr[2] * (1.0 + 0.01 * c * rng.standard_normal(csr[2].shape[0]))
            systems.append(((csr[0], csr[1], v), mis))
    for seed in range(40):
        (csr, a) = _random_csr(int(20 + 5 * seed), 1000 + seed)
        systems.append((csr, np.random.default_rng(seed).normal(size=a.shape[0])))
    mats = [s[0] for s in systems]
    rhs = [s[1] for s in systems]
    copies = [(m[0].copy(), m[1].copy(), m[2].copy()) for m in mats], [r.copy() for r in rhs]
    solver = CudaSparseLinearSolver()
    errors = [None] * len(mats)
    xs = solver.solve_batch(mats, rhs, errors)
    assert all(e is None for e in errors)
    for (rp, ci, v), b, x in zip(mats, rhs, xs):
        ref = oracle.sparse_solve(rp, ci, v, b)
        assert ref is not None and x is not None
        assert np.max(np.abs(x - ref)) <= REL_TOL * max(1.0, np.max(np.abs(ref)))
    for m, c in zip(mats, copies[0]):  # inputs unmodified
        assert all(np.array_equal(p, q) for p, q in zip(m, c))
    assert all(np.array_equal(r, c) for r, c in zip(rhs, copies[1]))
    again = solver.solve_batch(mats, rhs)  # the analysed patterns are reused: same results bit for bit
    assert all(np.array_equal(a, b) for a, b in zip(xs, again))


@pytest.mark.gpu
def test_failures_stay_with_their_system():
    from gridsim_b200.engine import CudaSparseLinearSolver
    (rp, ci, v), a = _random_csr(30, 7)
    b = np.ones(30)
    sing = v.copy()
    sing[rp[3]:rp[4]] = 0.0  # a zero row: singular
    nan = v.copy()
    nan[0] = np.nan
    bad_ci = ci.copy()
    bad_ci[0] = 30  # a column out of range
    solver = CudaSparseLinearSolver()
    errors = [None] * 5
    xs = solver.solve_batch([(rp, ci, v), (rp, ci, sing), (rp, ci, nan), (rp, bad_ci, v), (rp, ci, v)],
                            [b, b, b, b, b], errors)
    ref = np.linalg.solve(a, b)
    assert np.max(np.abs(xs[0] - ref)) <= REL_TOL * np.max(np.abs(ref))
    assert xs[1] is None and errors[1] is None  # singular: no result, no exception (ISparseLinearSolver returns null)
    assert xs[2] is None and isinstance(errors[2], ValueError)
    assert xs[3] is None and isinstance(errors[3], ValueError)
    assert np.array_equal(xs[4], xs[0])
    with pytest.raises(ValueError):
        solver.solve((rp, ci, nan), b)
    assert solver.solve((rp, ci, sing), b) is None


def _permuted_triangular(n, seed):
    """A diagonally dominant lower-triangular matrix with its rows shuffled: a structurally zero diagonal whose one
    zero-free row order is the triangle's (the reference's row pivoting finds it too)."""
    rng = np.random.default_rng(seed)
    low = np.tril(np.where(rng.random((n, n)) < 0.15, rng.normal(size=(n, n)), 0.0), -1)
    low += np.diag(np.abs(low).sum(axis=1) + 1.0 + rng.random(n))
    a = low[rng.permutation(n)]
    rows, cols = np.nonzero(a)
    indptr = np.searchsorted(rows, np.arange(n + 1)).astype(np.int32)
    return (indptr, cols.astype(np.int32), a[rows, cols]), a


def test_oracle_solver_handles_zero_diagonals():
    for seed in range(10):
        (rp, ci, v), a = _permuted_triangular(8 + 5 * seed, seed)
        assert any(a[i, i] == 0 for i in range(a.shape[0]))
        b = np.random.default_rng(seed).normal(size=a.shape[0])
        x = oracle.sparse_solve(rp, ci, v, b)
        ref = np.linalg.solve(a, b)
        assert np.max(np.abs(x - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.gpu
def test_zero_diagonals_are_solved_through_a_row_transversal():
    """Patterns whose diagonal is structurally zero get a zero-free row order before the analysis."""
    from gridsim_b200.engine import CudaSparseLinearSolver
    mats, rhs, dense = [], [], []
    for seed in range(12):
        (csr, a) = _permuted_triangular(10 + 7 * seed, 500 + seed)
        mats.append(csr)
        dense.append(a)
        rhs.append(np.random.default_rng(seed).normal(size=a.shape[0]))
    perm = np.random.default_rng(3).permutation(9)   # a permutation matrix: x = P^T b
    pm = np.zeros((9, 9))
    pm[np.arange(9), perm] = 1.0
    mats.append((np.arange(10, dtype=np.int32), perm.astype(np.int32), np.ones(9)))
    dense.append(pm)
    rhs.append(np.arange(1.0, 10.0))
    solver = CudaSparseLinearSolver()
    errors = [None] * len(mats)
    xs = solver.solve_batch(mats, rhs, errors)
    assert all(e is None for e in errors)
    for (rp, ci, v), b, a, x in zip(mats, rhs, dense, xs):
        ref = oracle.sparse_solve(rp, ci, v, b)
        assert x is not None and ref is not None
        assert np.max(np.abs(x - ref)) <= REL_TOL * max(1.0, np.max(np.abs(ref)))
        assert np.max(np.abs(a @ x - b)) <= 1e-9 * max(1.0, np.max(np.abs(b)))
    # no zero-free row order exists (column 0 is empty): singular, as the reference reports it
    rp = np.array([0, 1, 2, 4], np.int32)
    ci = np.array([1, 2, 1, 2], np.int32)
    assert solver.solve((rp, ci, np.array([1.0, 2.0, 3.0, 4.0])), np.ones(3)) is None


def _csr_of(a):
    a = np.asarray(a, float)
    rows, cols = np.nonzero(a)
    indptr = np.searchsorted(rows, np.arange(a.shape[0] + 1)).astype(np.int32)
    return indptr, cols.astype(np.int32), a[rows, cols]


def test_oracle_pivot_floor_is_per_row():
    """Gr044RowRelativePivotFloorTests.cs:85-100: diag(1e6, 1e-9) is well conditioned row by row (row 1's floor is
    1e-21), so the sparse LU solves it, bit for bit 1 / 1e6 and 1 / 1e-9."""
    x = oracle.sparse_solve(*_csr_of([[1e6, 0.0], [0.0, 1e-9]]), [1.0, 1.0])
    assert x is not None
    assert x[0] == 1.0 / 1e6 and x[1] == 1.0 / 1e-9


def test_oracle_pivot_floor_boundary():
    """Gr044RowRelativePivotFloorTests.cs:143-157: [[1, 0], [1, p]] with row 1's scale 1, so its floor is exactly
    1e-12 (NumericTolerances.PivotFloor(1.0)): p at the floor is singular, the next double above it is not."""
    at_floor = 1e-12 * 1.0
    above = np.nextafter(at_floor, np.inf)
    assert oracle.sparse_solve(*_csr_of([[1.0, 0.0], [1.0, at_floor]]), [1.0, 1.0]) is None
    x = oracle.sparse_solve(*_csr_of([[1.0, 0.0], [1.0, above]]), [1.0, 2.0])
    assert x is not None
    assert x[0] == 1.0 and x[1] == (2.0 - 1.0) / above


def test_oracle_near_singular_row_in_small_units_is_refused():
    """Gr044RowRelativePivotFloorTests.cs:170-176: row 1 has scale 1 and its pivot 1e-13 is below its own 1e-12
    floor."""
    assert oracle.sparse_solve(*_csr_of([[1e6, 0.0], [1.0, 1e-13]]), [1.0, 1.0]) is None


NR_DENSE = np.array([[4.0, -1.0, 0.5], [-1.0, 5.0, -2.0], [0.5, -2.0, 6.0]])
NR_RHS = np.array([1.0, -2.5, 0.75])


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_oracle_refuses_a_non_finite_right_hand_side(bad):
    """NonFiniteRightHandSideTests.cs:43-51: the sparse LU refuses a NaN or infinite right-hand side (an
    ArgumentException after the factorisation) instead of returning a non-finite solution."""
    b = NR_RHS.copy()
    b[2] = bad
    with pytest.raises(ValueError):
        oracle.sparse_solve(*_csr_of(NR_DENSE), b)


def test_oracle_singular_matrix_returns_none_whatever_its_right_hand_side():
    """NonFiniteRightHandSideTests.cs:53-66: the factorisation comes first, so a singular matrix returns null even
    with a NaN in b; and the finite solve is unchanged."""
    assert oracle.sparse_solve(*_csr_of([[1.0, 1.0], [1.0, 1.0]]), [np.nan, 1.0]) is None
    x = oracle.sparse_solve(*_csr_of(NR_DENSE), NR_RHS)
    assert np.max(np.abs(NR_DENSE @ x - NR_RHS)) < 1e-14


@pytest.mark.gpu
def test_non_finite_right_hand_side_is_checked_after_the_factorisation():
    """The same contract through the batched solve: in one call a singular matrix with a NaN right-hand side gives no
    result and no error (null), a regular one with an infinite right-hand side its refusal (ValueError), and the
    systems beside them are solved as alone; the bad systems' x are not written."""
    from gridsim_b200.engine import CudaSparseLinearSolver
    sing = _csr_of([[1.0, 1.0], [1.0, 1.0]])
    reg2 = _csr_of([[3.0, 1.0], [1.0, 2.0]])
    good = _csr_of(NR_DENSE)
    b_nan = np.array([np.nan, 1.0])
    b_inf = np.array([1.0, np.inf])
    solver = CudaSparseLinearSolver()
    errors = [None] * 4
    xs = solver.solve_batch([sing, reg2, good, reg2], [b_nan, b_inf, NR_RHS, np.array([4.0, 3.0])], errors)
    assert xs[0] is None and errors[0] is None
    assert xs[1] is None and isinstance(errors[1], ValueError)
    assert errors[2] is None and np.max(np.abs(NR_DENSE @ xs[2] - NR_RHS)) < 1e-12
    assert errors[3] is None and np.allclose(xs[3], [1.0, 1.0], rtol=0, atol=1e-14)
    with pytest.raises(ValueError):
        oracle.sparse_solve(*reg2, b_inf)
    assert oracle.sparse_solve(*sing, b_nan) is None
