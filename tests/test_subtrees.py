"""The subtree schedule of the factorisation (gs::BuildSubtrees) on the CPU: its precondition, that every task of a
subtree reads only values written by tasks of the same subtree at earlier stages, checked on the 2,000-bus grid at
several cuts, with a small C++ harness compiled from the engine's host sources against the symbolic analysis."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from gridsim_b200 import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gridsim_b200", "csrc")

HARNESS = r'''
#include <algorithm>
#include <vector>
#include "gs_host.h"
// returns the number of operand reads whose writer is in another subtree or at a later or equal stage; *nSub gets
// the subtree count and *nTasks the tasks below the cut
extern "C" long check_subtrees(const gs_grid_desc* d, int cut, int* nSub, long* nTasks) {
    gs::HostGrid g;
    if (!gs::CopyGrid(d, g).empty()) return -1;
    gs::Symbolic s;
    if (!gs::Analyze(g, s).empty()) return -2;
    const auto& P = s.ps;
    if (!P.on) return -3;
    gs::SubtreeSchedule st = gs::BuildSubtrees(s, cut);
    const size_t nT = P.taskA.size() / 4;
    std::vector<int> subOf(nT, -1), stageOf(nT, -1);
    long tasks = 0;
    for (int t = 0; t < st.nSub; t++)
        for (int q = st.subStage[t]; q < st.subStage[t + 1]; q++)
            for (int w = st.stagePtr[q]; w < st.stagePtr[q + 1]; w++) {
                const int task = P.factor.work[st.work[w]];
                subOf[task] = t;
                stageOf[task] = q;
                tasks++;
            }
    // the task writing each LU slot and each right-hand-side entry
    std::vector<int> wSlot(s.nnzLU, -1), wY(s.m, -1);
    for (size_t t = 0; t < nT; t++) {
        const int kind = P.taskA[4 * t + 2] & 7, k = P.taskA[4 * t + 3];
        const int s0 = P.taskB[4 * t], s1 = P.taskB[4 * t + 1], c = P.taskB[4 * t + 2];
        if (kind == gs::kFwd) wY[s0] = (int)t;
        else if (kind == gs::kPFwd) { wY[k] = (int)t; wY[k + 1] = (int)t; }
        else if (kind == gs::kPDiag) { wSlot[s0 + 1] = (int)t; wSlot[s0 + 2 + c] = (int)t; }
        else if (kind == gs::kPUpper || kind == gs::kPLower) { wSlot[s0] = (int)t; wSlot[s1] = (int)t; }
        else if (kind != gs::kDiag) wSlot[s0] = (int)t;
    }
    long bad = 0;
    for (size_t t = 0; t < nT; t++) {
        if (subOf[t] < 0) continue;
        const int kind = P.taskA[4 * t + 2] & 7;
        const bool rhs = kind == gs::kFwd || kind == gs::kPFwd;
        const bool l1 = kind == gs::kPDiag || kind == gs::kPUpper || kind == gs::kPFwd;
        const bool r1 = kind == gs::kPDiag || kind == gs::kPLower;
        for (int q = P.taskA[4 * t]; q < P.taskA[4 * t + 1]; q++) {
            const int a = P.pairs[2 * q], c = P.pairs[2 * q + 1];
            int ws[4] = {wSlot[a], l1 ? wSlot[a + 1] : -1, rhs ? wY[c] : wSlot[c], (!rhs && r1) ? wSlot[c + 1] : -1};
            for (int w : ws)
                if (w >= 0 && (subOf[w] != subOf[t] || stageOf[w] >= stageOf[t])) bad++;
        }
    }
    *nSub = st.nSub;
    *nTasks = tasks;
    return bad;
}
'''


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("subtrees")
    src = d / "harness.cpp"
    src.write_text(HARNESS)
    lib = d / "libharness.so"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", str(lib), str(src),
                           os.path.join(CSRC, "gs_host.cpp"), os.path.join(CSRC, "gs_symbolic.cpp")])
    h = ctypes.CDLL(str(lib))
    h.check_subtrees.restype = ctypes.c_long
    return h


@pytest.mark.parametrize("cut", [0, 2, 4, 12, 30])
def test_subtree_tasks_read_only_their_own_subtree(harness, cut):
    m = synthetic.config_grid(1, 0)
    d = m.desc()
    n_sub = ctypes.c_int()
    n_tasks = ctypes.c_long()
    bad = harness.check_subtrees(ctypes.byref(d), cut, ctypes.byref(n_sub), ctypes.byref(n_tasks))
    assert bad == 0
    assert n_sub.value > 0 and n_tasks.value > 0
