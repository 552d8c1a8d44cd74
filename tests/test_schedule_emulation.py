"""The factorisation and triangular-solve schedules of the symbolic analysis, run on the CPU the way the device runs
them: phase by phase (the level kernels' launches), every task of a phase reading only the values from before the
phase, so that a dependency between two tasks of one phase (a read the device may race with) changes the result.

A small C++ harness, compiled from the engine's host sources, analyses a grid (gs::Analyze, with and without the
Q-limit superset pattern) or a bare matrix (gs::AnalyzeMatrix, the batched linear seam), fills the matrix cells with a
random diagonally dominant matrix and every fill slot with 1e30 (so a wrong "starts from A" bit shows), and runs:

* the paired schedule (2 x 2 units: kPDiag / kPUpper / kPLower / kPFwd and single-node entries) and the scalar one;
* the one-system walks' top part (FP64 and FP32 budgets): the levels below it on the scalar schedule, the top loaded
  into a shared-memory image with its external pairs applied, walked there phase by phase and stored back;
* the fused factorisation + forward substitution, then the backward substitution level by level from the root;
* the forward-only schedule of a second right-hand side (the mixed-precision refinement's solve);
* the factorisation with a subtree cut: the subtrees below the cut each alone, stage by stage (k_psubtree), then the
  paired schedule's levels above it.

Each solve must leave |A x - b| at rounding level; no LU slot, pivot or right-hand-side entry may be written twice in
one factorisation, and no pivot may collapse. The task semantics restate the device's (gs_paired.cuh pkFactorTask,
pkForwardTask, pkBackTask; gs_kernels.cuh for the scalar entries) in plain sequential C++."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from gridsim_b200 import synthetic
from conftest import golden_model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gridsim_b200", "csrc")

HARNESS = r'''
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>
#include "gs_host.h"

namespace {
using gs::Symbolic;

struct Out {
    double resid;       // max |A x - b| / max |b| of the fused factor + forward, then backward
    double residFwd;    // the same through the forward-only schedule of a second right-hand side
    int64_t rewrites;   // LU slots, pivots or right-hand-side entries written more than once in one factorisation
    int64_t perturbed;  // pivots at or below their floor
    int32_t phases;     // factorisation phases run
    int32_t paired;     // 1 when the paired schedule ran
    int32_t topLevels;  // levels walked in the top part's shared-memory image
    int64_t itemErrors; // violations of the item structure the kernels rely on (CheckItems)
};

struct Emu {
    const Symbolic& s;
    std::vector<double> lu, piv, y;               // live values
    std::vector<double> L, Pv, Y;                 // the values before the phase
    std::vector<int> wLu, wPiv, wY;
    int64_t perturbed = 0;
    explicit Emu(const Symbolic& sym) : s(sym) {}
    void snap() { L = lu; Pv = piv; Y = y; }
    void putLu(int64_t i, double v) { lu[i] = v; wLu[i]++; }
    void putY(int64_t i, double v) { y[i] = v; wY[i]++; }
    void putPiv(int i, double v) { piv[i] = v; wPiv[i]++; }
    double pivot(double a, double v) {  // the FP64 floor of the device (1e-12 x max(1, |a|))
        const double fl = 1e-12 * std::max(1.0, std::fabs(a));
        if (!(std::fabs(v) > fl)) { perturbed++; v = v < 0 ? -fl : fl; }
        return v;
    }
};

// the products of pairs [q0, q1) (K as on the device: 1 single, 2 left pair, 3 right pair, 4 block)
void Sums(const std::vector<int32_t>& pr, int64_t q0, int64_t q1, int K, const std::vector<double>& Lv,
          const std::vector<double>& R, double acc[4]) {
    acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
    for (int64_t q = q0; q < q1; q++) {
        const int a = pr[2 * q], c = pr[2 * q + 1];
        const double l0 = Lv[a], r0 = R[c];
        acc[0] += l0 * r0;
        if (K == 2) acc[1] += Lv[a + 1] * r0;
        if (K == 3) acc[1] += l0 * R[c + 1];
        if (K == 4) { acc[1] += l0 * R[c + 1]; acc[2] += Lv[a + 1] * r0; acc[3] += Lv[a + 1] * R[c + 1]; }
    }
}

// a single node's entry (kDiag, kUpper, kFwd, kLower) of either schedule
void Entry(Emu& e, int kind, bool hasA, int k, int64_t slot, const std::vector<int32_t>& pr, int64_t q0, int64_t q1) {
    double acc[4];
    const bool fwd = kind == gs::kFwd;
    const double a = fwd ? e.Y[slot] : (hasA ? e.L[slot] : 0.0);
    Sums(pr, q0, q1, 1, e.L, fwd ? e.Y : e.L, acc);
    double v = a - acc[0];
    if (kind == gs::kDiag) { e.putPiv(k, e.pivot(a, v)); return; }
    if (kind == gs::kLower) v = v / e.Pv[k];
    if (fwd) e.putY(slot, v); else e.putLu(slot, v);
}

// one task of the paired factorisation (pkFactorTask)
void PairTask(Emu& e, const Symbolic::PairSchedule& P, int t) {
    const int32_t* A = &P.taskA[4 * (size_t)t];
    const int32_t* D = &P.taskB[4 * (size_t)t];
    const int kind = A[2] & 7, k = A[3];
    auto has = [&](int i) { return ((A[2] >> (3 + i)) & 1) != 0; };
    if (kind < 4) { Entry(e, kind, has(0), k, D[0], P.pairs, A[0], A[1]); return; }
    double acc[4];
    if (kind == gs::kPDiag) {
        const int64_t bk = D[0], bk1 = D[1], c = D[2];
        const double a00 = has(0) ? e.L[bk] : 0.0, a01 = has(1) ? e.L[bk + 1] : 0.0;
        const double a10 = has(2) ? e.L[bk + 2 + c] : 0.0, a11 = has(3) ? e.L[bk1] : 0.0;
        Sums(P.pairs, A[0], A[1], 4, e.L, e.L, acc);
        const double p0 = e.pivot(a00, a00 - acc[0]);
        const double u01 = a01 - acc[1];
        const double l10 = (a10 - acc[2]) / p0;
        const double p1 = e.pivot(a11, a11 - acc[3] - l10 * u01);
        e.putPiv(k, p0);
        e.putLu(bk + 1, u01);
        e.putLu(bk + 2 + c, l10);
        e.putPiv(k + 1, p1);
        return;
    }
    if (kind == gs::kPUpper) {
        const double a0 = has(0) ? e.L[D[0]] : 0.0, a1 = has(1) ? e.L[D[1]] : 0.0, l10 = e.L[D[2]];
        Sums(P.pairs, A[0], A[1], 2, e.L, e.L, acc);
        const double v0 = a0 - acc[0];
        e.putLu(D[0], v0);
        e.putLu(D[1], a1 - acc[1] - l10 * v0);
        return;
    }
    if (kind == gs::kPLower) {
        const double a0 = has(0) ? e.L[D[0]] : 0.0, a1 = has(1) ? e.L[D[1]] : 0.0;
        const double u01 = e.L[D[2]], p0 = e.Pv[k], p1 = e.Pv[k + 1];
        Sums(P.pairs, A[0], A[1], 3, e.L, e.L, acc);
        const double v0 = (a0 - acc[0]) / p0;
        e.putLu(D[0], v0);
        e.putLu(D[1], (a1 - acc[1] - v0 * u01) / p1);
        return;
    }
    // kPFwd
    const double y0 = e.Y[k], y1 = e.Y[k + 1], l10 = e.L[D[2]];
    Sums(P.pairs, A[0], A[1], 2, e.L, e.Y, acc);
    const double v0 = y0 - acc[0];
    e.putY(k, v0);
    e.putY(k + 1, y1 - acc[1] - l10 * v0);
}

// forward-only task (pkForwardTask): the factorisation's forward entries on a second right-hand side in e.y
void PairForward(Emu& e, const Symbolic::PairSchedule& P, int t) {
    const int32_t* A = &P.taskA[4 * (size_t)t];
    const int32_t* D = &P.taskB[4 * (size_t)t];
    double acc[4];
    if ((A[2] & 7) == gs::kFwd) {
        Sums(P.pairs, A[0], A[1], 1, e.L, e.Y, acc);
        e.y[D[0]] = e.Y[D[0]] - acc[0];
        return;
    }
    const int k = A[3];
    const double y0 = e.Y[k], y1 = e.Y[k + 1], l10 = e.L[D[2]];
    Sums(P.pairs, A[0], A[1], 2, e.L, e.Y, acc);
    const double v0 = y0 - acc[0];
    e.y[k] = v0;
    e.y[k + 1] = y1 - acc[1] - l10 * v0;
}

// backward task of a unit (pkBackTask) on x = e.y
void PairBack(Emu& e, const Symbolic::PairSchedule& P, int t) {
    const int32_t* A = &P.bTaskA[4 * (size_t)t];
    const int32_t* D = &P.bTaskB[4 * (size_t)t];
    const int k = A[3];
    const bool pair = A[2] == gs::kBPair;
    const int64_t s0 = pair ? D[0] : (int64_t)D[0] + 1, s1 = D[1];
    double a0 = 0.0, a1 = 0.0;
    for (int r = A[0]; r < A[1]; r++) {
        const double xr = e.Y[e.s.pRows[r]];
        a0 += e.lu[s0 + (r - A[0])] * xr;
        if (pair) a1 += e.lu[s1 + (r - A[0])] * xr;
    }
    if (!pair) { e.y[k] = (e.Y[k] - a0) / e.piv[k]; return; }
    const double v1 = (e.Y[k + 1] - a1) / e.piv[k + 1];
    e.y[k + 1] = v1;
    e.y[k] = (e.Y[k] - e.lu[D[2]] * v1 - a0) / e.piv[k];
}

// backward substitution of a single node on the scalar schedule
void NodeBack(Emu& e, int k) {
    const Symbolic& s = e.s;
    double a = 0.0;
    for (int t = 0; t < s.pRowPtr[k + 1] - s.pRowPtr[k]; t++)
        a += e.lu[s.luBase[k] + 1 + t] * e.Y[s.pRows[s.pRowPtr[k] + t]];
    e.y[k] = (e.Y[k] - a) / e.piv[k];
}

// phases [from, nPh) of a schedule (nPh < 0: to the last), in order or from the last one down
template <class F>
void RunPhases(Emu& e, const Symbolic::Schedule& sc, bool reverse, F task, int nPh = -1, int from = 0) {
    if (nPh < 0) nPh = (int)sc.levelWorkPtr.size() - 1;
    for (int i = from; i < nPh; i++) {
        const int ph = reverse ? nPh - 1 - (i - from) : i;
        e.snap();
        for (int w = sc.levelWorkPtr[ph]; w < sc.levelWorkPtr[ph + 1]; w++) task(sc.work[w]);
    }
}

// The one-system walks' top part (factorSystem / backwardSystem / forwardSystem): the levels from L0 up held in a
// shared-memory image `sm`, loaded from global memory with the external pairs applied, walked phase by phase (every
// entry of a phase reading the image from before the phase), stored back. Every image value starts as 1e30, so a
// value read before it is loaded shows.
struct TopEmu {
    Emu& e;
    const Symbolic::TopPart& t;
    std::vector<double> sm, S;
    TopEmu(Emu& em, const Symbolic::TopPart& tp) : e(em), t(tp) {}
    double ext(int ti, const std::vector<double>& rhs, bool fwd) {
        double acc = 0.0;
        for (int q = t.extPtr[ti]; q < t.extPtr[ti + 1]; q++)
            acc += e.lu[t.extPairs[2 * q]] * (fwd ? rhs[t.extPairs[2 * q + 1]] : e.lu[t.extPairs[2 * q + 1]]);
        return acc;
    }
    double dot(int ti) {
        double acc = 0.0;
        for (int q = t.intPtr[ti]; q < t.intPtr[ti + 1]; q++) acc += S[t.intPairs[2 * q]] * S[t.intPairs[2 * q + 1]];
        return acc;
    }
    void load(const std::vector<int32_t>& list, const std::vector<double>& rhs) {
        const Symbolic& s = e.s;
        for (int ti : list) {
            const int en = t.ent[ti];
            const bool fwd = s.entKind[en] == gs::kFwd;
            const double base = fwd ? rhs[s.entNode[en]] : (s.entHasA[en] ? e.lu[s.entSlot[en]] : 0.0);
            sm[t.entSm[ti]] = base - ext(ti, rhs, fwd);
        }
    }
    void factor() {
        const Symbolic& s = e.s;
        sm.assign(t.nSlots + t.nNodes, 1e30);
        load(t.loadList, e.y);
        const int nTop = s.nLevels - t.L0;
        for (int i = 0; i < 2 * nTop; i++) {
            S = sm;
            for (int w = t.fWalkPtr[i]; w < t.fWalkPtr[i + 1]; w++) {
                const int ti = t.fWalk[w], en = t.ent[ti], idx = t.entSm[ti], kind = s.entKind[en];
                double v = S[idx] - dot(ti);
                if (kind == gs::kDiag) v = e.pivot(s.entHasA[en] ? e.lu[s.entSlot[en]] : 0.0, v);
                else if (kind == gs::kLower) v = v / S[t.smemBase[s.entNode[en]]];
                sm[idx] = v;
            }
        }
        for (int q = 0; q < t.nSlots; q++) {
            if (t.slotDiagNode[q] >= 0) e.putPiv(t.slotDiagNode[q], sm[q]);
            else e.putLu(t.slotGlobal[q], sm[q]);
        }
        for (int i = 0; i < t.nNodes; i++) e.putY(t.nodes[i], sm[t.nSlots + i]);
    }
    void backward() {
        const Symbolic& s = e.s;
        sm.assign(t.nSlots + t.nNodes, 1e30);
        for (int q = 0; q < t.nSlots; q++)
            sm[q] = t.slotDiagNode[q] >= 0 ? e.piv[t.slotDiagNode[q]] : e.lu[t.slotGlobal[q]];
        for (int i = 0; i < t.nNodes; i++) sm[t.nSlots + i] = e.y[t.nodes[i]];
        for (int lt = s.nLevels - t.L0 - 1; lt >= 0; lt--) {
            S = sm;
            for (int w = t.bWalkPtr[lt]; w < t.bWalkPtr[lt + 1]; w++) {
                const int ni = t.bWalk[w], k = t.nodes[ni], base = t.smemBase[k], c = s.luCnt[k];
                double acc = 0.0;
                for (int u = 0; u < c; u++) acc += S[base + 1 + u] * S[t.bRowSm[t.bRowPtr[ni] + u]];
                sm[t.nSlots + ni] = (S[t.nSlots + ni] - acc) / S[base];
            }
        }
        for (int i = 0; i < t.nNodes; i++) e.y[t.nodes[i]] = sm[t.nSlots + i];
    }
    void forward() {
        const Symbolic& s = e.s;
        sm.assign(t.nSlots + t.nNodes, 1e30);
        for (int q = 0; q < t.nSlots; q++) sm[q] = e.lu[t.slotGlobal[q]];
        load(t.fwdLoadList, e.y);
        for (int lt = 0; lt < s.nLevels - t.L0; lt++) {
            S = sm;
            for (int w = t.vWalkPtr[lt]; w < t.vWalkPtr[lt + 1]; w++) sm[t.entSm[t.vWalk[w]]] = S[t.entSm[t.vWalk[w]]] - dot(t.vWalk[w]);
        }
        for (int i = 0; i < t.nNodes; i++) e.y[t.nodes[i]] = sm[t.nSlots + i];
    }
};

// The item structure the kernels rely on, per phase of a schedule: items cover the phase's work in order; the wide
// ones (count -1, one piece for the whole warp) come first, levelWide of them; the others hold 1 .. 8 pieces (a warp's
// lane groups), each short enough for a lane group's one round of loads (at most 32 index pairs or rows), ordered
// longest first, with levelMid of them longer than `midAbove`. `len` gives a piece's length as the packing measured it,
// `raw` its index pairs (or rows). Returns the number of violations.
template <class Len, class Raw>
int64_t CheckItems(const Symbolic::Schedule& sc, int midAbove, Len len, Raw raw) {
    int64_t bad = 0;
    const int nPh = (int)sc.levelWorkPtr.size() - 1;
    if ((int)sc.levelItemPtr.size() != nPh + 1 || (int)sc.levelWide.size() != nPh || (int)sc.levelMid.size() != nPh)
        return 1;
    for (int ph = 0; ph < nPh; ph++) {
        int w = sc.levelWorkPtr[ph], wide = 0, mid = 0;
        bool inShort = false;
        int64_t prev = INT64_MAX;
        for (int it = sc.levelItemPtr[ph]; it < sc.levelItemPtr[ph + 1]; it++) {
            const int start = sc.items[2 * it], count = sc.items[2 * it + 1];
            if (start != w) bad++;
            if (count < 0) {
                if (inShort) bad++;
                if (len(sc.work[start]) <= 32) bad++;
                wide++;
                w++;
                continue;
            }
            inShort = true;
            if (count < 1 || count > 8) bad++;
            for (int q = start; q < start + count; q++) {
                const int64_t l = len(sc.work[q]);
                if (l > 32 || raw(sc.work[q]) > 32 || l > prev) bad++;
                if (l > midAbove) mid++;
                prev = l;
            }
            w += std::max(count, 0);
        }
        if (w != sc.levelWorkPtr[ph + 1] || wide != sc.levelWide[ph] || mid != sc.levelMid[ph]) bad++;
    }
    return bad;
}

int64_t CheckAllItems(const Symbolic& s) {
    int64_t bad = 0;
    auto ePairs = [&](int e) { return s.entPairPtr[e + 1] - s.entPairPtr[e]; };
    bad += CheckItems(s.factor, 8, ePairs, ePairs);
    bad += CheckItems(s.forward, 8, ePairs, ePairs);
    auto nRows = [&](int q) { return (int64_t)s.luCnt[s.levelNodes[q]]; };
    bad += CheckItems(s.backward, 8, nRows, nRows);
    const Symbolic::PairSchedule& P = s.ps;
    if (P.on) {
        auto tPairs = [&](int t) { return (int64_t)P.taskA[4 * (size_t)t + 1] - P.taskA[4 * (size_t)t]; };
        auto tLen = [&](int t) { return ((P.taskA[4 * (size_t)t + 2] & 7) == gs::kPDiag ? 2 : 1) * tPairs(t); };
        bad += CheckItems(P.factor, 4, tLen, tPairs);
        bad += CheckItems(P.forward, 4, tPairs, tPairs);
        auto bRows = [&](int t) { return (int64_t)P.bTaskA[4 * (size_t)t + 1] - P.bTaskA[4 * (size_t)t]; };
        bad += CheckItems(P.backward, 4, bRows, bRows);
    }
    return bad;
}

double Residual(const Symbolic& s, const std::vector<double>& a, const std::vector<double>& x,
                const std::vector<double>& b) {
    std::vector<double> r(b);
    for (int l = 0; l < s.m; l++)
        for (int p = s.aColPtr[l]; p < s.aColPtr[l + 1]; p++) r[s.aRow[p]] -= a[s.aSlot[p]] * x[l];
    double num = 0.0, den = 0.0;
    for (int i = 0; i < s.m; i++) { num = std::max(num, std::fabs(r[i])); den = std::max(den, std::fabs(b[i])); }
    return num / den;
}

// mode 0: the scalar schedule; 1: the paired one; 2 / 3: the scalar one below the FP64 / FP32 top part, the top
// part walked as the one-system kernels walk it; 4: the paired one with the subtrees below unit level `cut` factored
// first (k_psubtree: each subtree alone, stage by stage), then the levels above the cut
int Emulate(const Symbolic& s, int mode, uint64_t seed, Out* out, int cut = -1) {
    const Symbolic::PairSchedule& P = s.ps;
    const bool usePaired = mode == 1 || mode == 4;
    if (usePaired && !P.on) return -3;
    const Symbolic::TopPart* tp = (mode == 2 || mode == 3) ? &s.top[mode - 2] : nullptr;
    const bool top = tp && tp->L0 < s.nLevels;
    const int L0 = top ? tp->L0 : s.nLevels;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    // a random row diagonally dominant matrix on the matrix's own cells; every other slot holds 1e30
    std::vector<double> a(s.nnzLU, 1e30), rowAbs(s.m, 0.0);
    std::vector<int64_t> diag(s.m, -1);
    for (int l = 0; l < s.m; l++)
        for (int p = s.aColPtr[l]; p < s.aColPtr[l + 1]; p++) {
            if (s.aRow[p] == l) { diag[l] = s.aSlot[p]; continue; }
            const double v = U(rng);
            a[s.aSlot[p]] = v;
            rowAbs[s.aRow[p]] += std::fabs(v);
        }
    for (int k = 0; k < s.m; k++) {
        if (diag[k] < 0) return -4;
        a[diag[k]] = (rowAbs[k] + 1.0) * (U(rng) < 0.0 ? -1.0 : 1.0);
    }
    std::vector<double> b(s.m), b2(s.m);
    for (auto& v : b) v = U(rng);
    for (auto& v : b2) v = U(rng);

    Emu e(s);
    e.lu = a;
    e.piv.assign(s.m, 0.0);
    e.y = b;
    e.wLu.assign(s.nnzLU, 0);
    e.wPiv.assign(s.m, 0);
    e.wY.assign(s.m, 0);
    if (mode == 4) {
        const gs::SubtreeSchedule st = gs::BuildSubtrees(s, cut);
        if (st.nSub <= 0) return -5;
        for (int sub = 0; sub < st.nSub; sub++)
            for (int q = st.subStage[sub]; q < st.subStage[sub + 1]; q++) {
                e.snap();
                for (int w = st.stagePtr[q]; w < st.stagePtr[q + 1]; w++) PairTask(e, P, P.factor.work[st.work[w]]);
            }
        RunPhases(e, P.factor, false, [&](int t) { PairTask(e, P, t); }, -1, 2 * (cut + 1));
    } else if (usePaired) {
        RunPhases(e, P.factor, false, [&](int t) { PairTask(e, P, t); });
    } else {
        RunPhases(e, s.factor, false, [&](int en) {
            Entry(e, s.entKind[en], s.entHasA[en] != 0, s.entNode[en], s.entSlot[en], s.pairs, s.entPairPtr[en],
                  s.entPairPtr[en + 1]);
        }, 2 * L0);
    }
    TopEmu te(e, top ? *tp : s.top[0]);
    if (top) te.factor();
    out->phases = usePaired ? (int)P.factor.levelWorkPtr.size() - 1 : 2 * s.nLevels;
    out->topLevels = s.nLevels - L0;
    int64_t rewrites = 0;
    for (int v : e.wLu) rewrites += v > 1;
    for (int v : e.wY) rewrites += v > 1;
    for (int v : e.wPiv) rewrites += v != 1;  // every pivot exactly once
    out->rewrites = rewrites;
    out->perturbed = e.perturbed;
    out->paired = usePaired ? 1 : 0;
    out->itemErrors = CheckAllItems(s);
    auto backward = [&]() {
        if (usePaired) { RunPhases(e, P.backward, true, [&](int t) { PairBack(e, P, t); }); return; }
        if (top) te.backward();
        RunPhases(e, s.backward, true, [&](int q) { NodeBack(e, s.levelNodes[q]); }, L0);
    };
    backward();
    out->resid = Residual(s, a, e.y, b);
    // a second right-hand side through the forward-only schedule, then the backward one
    e.y = b2;
    if (usePaired) {
        RunPhases(e, P.forward, false, [&](int t) { PairForward(e, P, t); });
    } else {
        RunPhases(e, s.forward, false, [&](int en) {
            double acc[4];
            Sums(s.pairs, s.entPairPtr[en], s.entPairPtr[en + 1], 1, e.L, e.Y, acc);
            e.y[s.entSlot[en]] = e.Y[s.entSlot[en]] - acc[0];
        }, L0);
        if (top) te.forward();
    }
    backward();
    out->residFwd = Residual(s, a, e.y, b2);
    return 0;
}
}  // namespace

extern "C" int emulate_grid(const gs_grid_desc* d, int qlim, int mode, unsigned long long seed, Out* out) {
    gs::HostGrid g;
    if (!gs::CopyGrid(d, g).empty()) return -1;
    Symbolic s;
    if (!gs::Analyze(g, s, qlim != 0).empty()) return -2;
    return Emulate(s, mode, seed, out);
}

extern "C" int emulate_grid_subtrees(const gs_grid_desc* d, int cut, unsigned long long seed, Out* out) {
    gs::HostGrid g;
    if (!gs::CopyGrid(d, g).empty()) return -1;
    Symbolic s;
    if (!gs::Analyze(g, s).empty()) return -2;
    return Emulate(s, 4, seed, out, cut);
}

extern "C" int emulate_matrix(int n, const int* rowPtr, const int* colIdx, int mode, unsigned long long seed,
                              Out* out) {
    Symbolic s;
    std::vector<int> aSlot;
    if (!gs::AnalyzeMatrix(n, rowPtr, colIdx, s, aSlot).empty()) return -2;
    return Emulate(s, mode, seed, out);
}
'''


class Out(ctypes.Structure):
    _fields_ = [("resid", ctypes.c_double), ("resid_fwd", ctypes.c_double), ("rewrites", ctypes.c_int64),
                ("perturbed", ctypes.c_int64), ("phases", ctypes.c_int32), ("paired", ctypes.c_int32),
                ("top_levels", ctypes.c_int32), ("item_errors", ctypes.c_int64)]

# the schedules run: the paired one, the scalar one, and the scalar one below the FP64 / FP32 top part
MODES = {"paired": 1, "scalar": 0, "top_fp64": 2, "top_fp32": 3}


# rounding level of a diagonally dominant solve of a few thousand unknowns in FP64
RESID_TOL = 1e-12


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("emulation")
    src = d / "harness.cpp"
    src.write_text(HARNESS)
    lib = d / "libemulation.so"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", str(lib), str(src),
                           os.path.join(CSRC, "gs_host.cpp"), os.path.join(CSRC, "gs_symbolic.cpp")])
    h = ctypes.CDLL(str(lib))
    h.emulate_grid.restype = ctypes.c_int
    h.emulate_matrix.restype = ctypes.c_int
    h.emulate_grid_subtrees.restype = ctypes.c_int
    return h


@pytest.fixture(scope="module")
def grid_2000():
    return synthetic.config_grid(1, 0)


def _check(out, mode):
    assert out.item_errors == 0
    assert out.rewrites == 0
    assert (out.top_levels > 0) == (mode >= 2)
    assert out.perturbed == 0
    assert out.phases > 0
    assert out.resid < RESID_TOL
    assert out.resid_fwd < RESID_TOL


@pytest.mark.parametrize("qlim", [0, 1])
@pytest.mark.parametrize("schedule", list(MODES))
@pytest.mark.parametrize("name", ["case9", "case118", "case300"])
def test_case_schedules_solve(harness, name, schedule, qlim):
    m, _ = golden_model(name)
    d = m.desc()
    out = Out()
    rc = harness.emulate_grid(ctypes.byref(d), qlim, MODES[schedule], 7, ctypes.byref(out))
    assert rc == 0
    _check(out, MODES[schedule])


@pytest.mark.parametrize("qlim", [0, 1])
@pytest.mark.parametrize("schedule", list(MODES))
def test_2000_bus_schedules_solve(harness, grid_2000, schedule, qlim):
    d = grid_2000.desc()
    out = Out()
    rc = harness.emulate_grid(ctypes.byref(d), qlim, MODES[schedule], 11, ctypes.byref(out))
    assert rc == 0
    _check(out, MODES[schedule])


def _random_pattern(n, per_row, symmetric, seed):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        cols = set(rng.choice(n, size=per_row, replace=False).tolist())
        cols.add(i)
        rows.append(cols)
    if symmetric:
        for i in range(n):
            for j in list(rows[i]):
                rows[j].add(i)
    row_ptr = [0]
    col = []
    for i in range(n):
        c = sorted(rows[i])
        col.extend(c)
        row_ptr.append(len(col))
    return np.asarray(row_ptr, np.int32), np.asarray(col, np.int32)


@pytest.mark.parametrize("n,per_row,symmetric,seed", [(1, 0, False, 0), (2, 1, False, 1), (40, 2, False, 2),
                                                       (300, 3, True, 3), (600, 2, False, 4), (1500, 3, False, 5)])
def test_matrix_schedules_solve(harness, n, per_row, symmetric, seed):
    row_ptr, col = _random_pattern(n, per_row, symmetric, seed)
    for mode in MODES.values():
        out = Out()
        rc = harness.emulate_matrix(n, row_ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    col.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), mode, seed,
                                    ctypes.byref(out))
        if mode == 1 and rc == -3:  # no paired schedule for this pattern: the scalar one serves it
            continue
        assert rc == 0
        _check(out, mode)


@pytest.mark.parametrize("cut", [0, 2, 4, 12, 30])
def test_2000_bus_subtrees_then_levels_solve(harness, grid_2000, cut):
    """The factorisation as it runs with a subtree cut: the subtrees below unit level `cut` each alone, stage by stage
    (one CTA per subtree and system group), then the paired schedule's levels above the cut."""
    d = grid_2000.desc()
    out = Out()
    rc = harness.emulate_grid_subtrees(ctypes.byref(d), cut, 13, ctypes.byref(out))
    assert rc == 0
    _check(out, 1)
