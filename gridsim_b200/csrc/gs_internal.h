// gs_internal.h — host-side data of the gridsim_b200 engine (not part of the C ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gridsim_b200.h"

namespace gs {

// The grid as handed over the ABI, copied (the library keeps no caller pointer).
struct HostGrid {
    int n = 0, ngen = 0, nbr = 0;
    double base = 100.0;
    std::vector<int> busId, busType;
    std::vector<double> pd, qd, gsh, bsh, vm, vaDeg, vmin, vmax;
    std::vector<int> genBus;
    std::vector<double> pg, qg, vg, qmin, qmax;
    std::vector<uint8_t> genOn;
    std::vector<int> brF, brT;
    std::vector<double> r, x, b, tap, shift, rateA;
    std::vector<uint8_t> brOn;
};

// Entry kinds of the fused factor + forward-substitution schedule.
enum EntryKind : int32_t { kDiag = 0, kUpper = 1, kFwd = 2, kLower = 3 };

// Shared symbolic analysis of one grid (SparseNewtonRaphsonPowerFlow.BuildY / BuildJacobianStructure,
// NewtonShell.BuildBusSpec / EquationPositions, then the static-pivot LU pattern and its schedule).
struct Symbolic {
    int n = 0, nbr = 0;
    // ---- Y-bus of the intact grid: CSR, cells summed in stamping order (branches, then shunts) ----
    int nnzY = 0;
    std::vector<int> yRowPtr, yCol;
    std::vector<double> yG, yB;
    // per branch: its 4 cells (ff, tt, ft, tf) as Y positions (-1 when out of service) and the cells'
    // values with the branch removed (G, B pairs), summed in the same order as a rebuilt Y would be
    std::vector<int> brCell;      // [4*nbr]
    std::vector<double> brRed;    // [8*nbr]
    std::vector<double> brStamp;  // [8*nbr] yff, ytt, yft, ytf (re, im) for line flows
    // ---- bus specification ----
    std::vector<int> type0, pPos, qPos;
    int m = 0, npv = 0, npq = 0;
    std::vector<double> pspec, qspec, vm0, va0;  // va0 radians
    // ---- Jacobian superset pattern and the minimum-degree order ----
    int nnzJ = 0;
    std::vector<int> jRowPtr, jCol;
    std::vector<int> perm;  // pivot step -> equation
    std::vector<int> pinv;  // equation -> pivot step
    // ---- LU structure, node-major: node k holds [diag, U(k,P_k) ..., L(P_k,k) ...] from luBase[k] ----
    std::vector<int64_t> luBase;
    std::vector<int> luCnt;
    std::vector<int> pRowPtr, pRows;  // P_k (sorted pivot steps > k), CSR over k
    std::vector<int> parent;
    int64_t nnzLU = 0;
    int64_t flops = 0;  // multiply-adds of one numeric factorisation (+ forward substitution)
    std::vector<int> ySlot;          // [4*nnzY] Y cell -> LU slot of H, N, M, L (-1 absent)
    std::vector<int> busP, busQ;     // bus -> pivot step of its P / Q equation (-1 none)
    // ---- schedule ----
    int nLevels = 0;
    std::vector<int> level;          // per node
    std::vector<int> levelNodePtr, levelNodes;   // nodes by level (for the backward substitution)
    std::vector<int32_t> entSlot;    // LU slot, or y index for kFwd
    std::vector<int32_t> entKind;
    std::vector<int32_t> entHasA;    // start from the filled Jacobian value
    std::vector<int64_t> entPairPtr; // [nEnt+1]
    std::vector<int32_t> pairs;      // 2 per pair: (left slot, right slot-or-y-index)
    std::vector<int32_t> diagPairNode; // per node: entry index of its diagonal
    std::vector<int32_t> entNode;    // node of each entry
    // Work schedules of the LU kernels. A schedule is a work list (entry or node indices) cut into items;
    // an item {start, count} is `count` short pieces of work done side by side by the lane groups of one
    // warp, or (count = -1) one long piece done by the whole warp. levelItemPtr cuts the items by level
    // (and, for the factorisation, by phase: 2 * level + 0 for diagonal / upper / forward entries, + 1 for
    // lower entries, which read the finished pivot).
    struct Schedule {
        std::vector<int32_t> work;
        std::vector<int32_t> items;        // 2 per item
        std::vector<int32_t> levelItemPtr;
        std::vector<int32_t> levelWorkPtr; // the work of a level (phase) is work[levelWorkPtr[i] .. [i+1])
        std::vector<int32_t> levelWide;    // how many of a level (phase)'s first items are wide (one piece each)
    };
    Schedule factor, backward, forward;
};

// Build the symbolic analysis; returns an empty string on success, else the reason.
std::string Analyze(const HostGrid& g, Symbolic& s);

// Minimum-degree order of a structurally symmetric pattern (pivot step -> index).
std::vector<int> MinimumDegreeOrder(int n, const std::vector<int>& rowPtr, const std::vector<int>& col);

}  // namespace gs
