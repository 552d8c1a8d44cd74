"""The engine's minimum-degree order (gs::MinimumDegreeOrder, run by the symbolic analysis) against the oracle's
restatement of the reference's SparseLu.Ordering (Numerics/MinimumDegreeOrdering.cs:23-121), on the CPU.

On a symmetric pattern the two are the same permutation: every Jacobian of the load flow (checked here on the golden
cases and the 2,000-bus grid, with the Jacobian patterns themselves equal), and symmetric bare matrices. So the
static pivots of the batched LU and the column order of the partial-pivoting re-solve are the reference's own order
for every Newton step. On a nonsymmetric bare matrix (the batched linear seam) the reference lists each node's
neighbours in the order a row-by-row scan meets them, which breaks minimum-degree ties differently; there the seam's
results agree with the reference's to rounding, not bit for bit."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle
from gridsim_b200 import synthetic
from tests.conftest import golden_model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gridsim_b200", "csrc")

HARNESS = r'''
#include <vector>
#include "gs_host.h"
// the analysed grid's equation count, its order (pivot step -> equation) and its Jacobian pattern (equation order)
extern "C" int engine_grid_order(const gs_grid_desc* d, int cap, int capNz, int* m, int* perm, int* rowPtr, int* col) {
    gs::HostGrid g;
    if (!gs::CopyGrid(d, g).empty()) return -1;
    gs::Symbolic s;
    if (!gs::Analyze(g, s).empty()) return -2;
    *m = s.m;
    if (s.m > cap || s.nnzJ > capNz) return -3;
    for (int i = 0; i < s.m; i++) perm[i] = s.perm[i];
    for (int i = 0; i <= s.m; i++) rowPtr[i] = s.jRowPtr[i];
    for (int i = 0; i < s.nnzJ; i++) col[i] = s.jCol[i];
    return 0;
}
// the order of a bare matrix's analysis (the batched linear seam)
extern "C" int engine_matrix_order(int n, const int* rp, const int* ci, int* perm) {
    gs::Symbolic s;
    std::vector<int> aSlot;
    if (!gs::AnalyzeMatrix(n, rp, ci, s, aSlot).empty()) return -2;
    for (int i = 0; i < n; i++) perm[i] = s.perm[i];
    return 0;
}
'''

P = ctypes.POINTER(ctypes.c_int)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("ordering")
    src = d / "harness.cpp"
    src.write_text(HARNESS)
    lib = d / "libordering.so"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", str(lib), str(src),
                           os.path.join(CSRC, "gs_host.cpp"), os.path.join(CSRC, "gs_symbolic.cpp")])
    return ctypes.CDLL(str(lib))


def _grid_order(h, m):
    cap, cap_nz = 20000, 400000
    perm, rp, col = np.zeros(cap, np.int32), np.zeros(cap + 1, np.int32), np.zeros(cap_nz, np.int32)
    mm = ctypes.c_int()
    d = m.desc()
    assert h.engine_grid_order(ctypes.byref(d), cap, cap_nz, ctypes.byref(mm), perm.ctypes.data_as(P),
                               rp.ctypes.data_as(P), col.ctypes.data_as(P)) == 0
    n = mm.value
    return perm[:n], rp[:n + 1], col[:rp[n]]


@pytest.mark.parametrize("name", ["case9", "case14", "case57", "case118", "case300", "grid2000"])
def test_jacobian_order_is_the_references(harness, name):
    m = synthetic.config_grid(1, 0) if name == "grid2000" else golden_model(name)[0]
    perm, rp, col = _grid_order(harness, m)
    orp, oci, _, _ = oracle.jacobian(m)
    assert np.array_equal(rp, orp) and np.array_equal(col, oci)
    assert np.array_equal(perm, oracle.md_order(orp, oci))


def _symmetric_pattern(n, per_row, seed):
    rng = np.random.default_rng(seed)
    rows = [set(rng.choice(n, size=per_row, replace=False).tolist()) | {i} for i in range(n)]
    for i in range(n):
        for j in list(rows[i]):
            rows[j].add(i)
    rp, col = [0], []
    for i in range(n):
        col.extend(sorted(rows[i]))
        rp.append(len(col))
    return np.asarray(rp, np.int32), np.asarray(col, np.int32)


@pytest.mark.parametrize("n,per_row,seed", [(1, 0, 0), (2, 1, 1), (50, 2, 2), (300, 3, 3), (1200, 2, 4)])
def test_symmetric_matrix_order_is_the_references(harness, n, per_row, seed):
    rp, ci = _symmetric_pattern(n, per_row, seed)
    perm = np.zeros(n, np.int32)
    assert harness.engine_matrix_order(n, rp.ctypes.data_as(P), ci.ctypes.data_as(P), perm.ctypes.data_as(P)) == 0
    assert np.array_equal(perm, oracle.md_order(rp, ci))
