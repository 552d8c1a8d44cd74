// gs_internal.h — host-side data of the gridsim_b200 engine (not part of the C ABI).
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <functional>
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
    std::vector<double> r, x, b, tap, shift, rateA, rateB, rateC;
    std::vector<uint8_t> brOn;
    // boundaries: members bndPtr[q] .. bndPtr[q+1]-1 (branch position, direction), limit in MW (0 = none)
    int nBnd = 0;
    std::vector<int> bndPtr, bndBranch, bndDir;
    std::vector<double> bndLimit;
    // voltage-dependent (ZIP) loads: [6 n] Ap Bp Cp Aq Bq Cq per bus, empty when every load is constant power
    std::vector<double> zip;
};

// Entry kinds of the fused factor + forward-substitution schedule.
enum EntryKind : int32_t { kDiag = 0, kUpper = 1, kFwd = 2, kLower = 3 };
// Task kinds of the paired schedule (Symbolic::PairSchedule): the entry kinds above for single nodes, then a pair's
// diagonal block, upper rows, lower columns and forward entry; backward tasks of a single node and of a pair.
enum PairTaskKind : int32_t { kPDiag = 4, kPUpper = 5, kPLower = 6, kPFwd = 7 };
enum PairBackKind : int32_t { kBNode = 0, kBPair = 1 };

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
    // per Y cell, its stamps in stamping order (owner branch, or -1 for a bus shunt, and the value): what a Y
    // rebuilt without a set of branches sums, cell by cell
    std::vector<int> ccPtr, ccOwner;
    std::vector<double> ccG, ccB;
    // ---- bus specification ----
    std::vector<int> type0, pPos, qPos;
    int m = 0, npv = 0, npq = 0;
    std::vector<double> pspec, qspec, vm0, va0;  // va0 radians
    // Q-limit enforcement (qlim): the Q equation of every PV bus is in the pattern; per-bus aggregate limits
    bool qlim = false;
    std::vector<double> qminMvar, qmaxMvar;
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
    // the matrix's own cells (the Jacobian's, or a loaded matrix's; fill left out) by column in pivot order: rows
    // aRow[aColPtr[l] .. aColPtr[l+1]) ascending, each with its LU slot; what the partial-pivoting re-solve reads
    std::vector<int32_t> aColPtr, aRow, aSlot;
    // the Jacobian pattern in equation order (jRowPtr / jCol) for the iterative fallback of a singular step: each
    // cell's LU slot, and the Y cell between its two buses (-1 within one bus), whose branch stamps decide whether the
    // cell exists in a system with branches out
    std::vector<int32_t> jSlot, jYcell;
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
        std::vector<int32_t> levelMid;     // how many of the short pieces after them are longer than 8 pairs
    };
    Schedule factor, backward, forward;

    // The paired schedule: two consecutive nodes k, k + 1 whose structure makes them one 2 x 2 block (a PQ bus's angle
    // and magnitude: parent(k) = k + 1, P_k = {k + 1} + P_{k+1}, and the row subtree of k + 1 is that of k plus k) form
    // one unit, every other node a unit of its own. A pair's entries are computed together, so that L(k + 1, j) =
    // L(k, j) + 1 slot and U(j, k + 1) = U(j, k) + 1 slot share one index pair and the elimination tree of units has
    // about half the levels. The LU storage is the node-major one above. Tasks (8 ints each, taskA / taskB):
    //   taskA = {first pair, end of pairs, kind | hasA bits << 3, node k}, taskB = {s0, s1, aux, 0} with
    //   kDiag / kUpper / kFwd / kLower (a single node's entries as above): s0 = slot (y index for kFwd);
    //   kPDiag: the 2 x 2 diagonal block, s0 = luBase[k], s1 = luBase[k + 1], aux = |P_{k+1}|, pairs (L(k, j), U(j, k));
    //   kPUpper: U(k, r), U(k + 1, r) in s0, s1, aux = slot of L(k + 1, k), pairs (L(k, j), U(j, r));
    //   kPLower: L(r, k), L(r, k + 1) in s0, s1, aux = slot of U(k, k + 1), pairs (L(r, j), U(j, k));
    //   kPFwd: y(k), y(k + 1), aux = slot of L(k + 1, k), pairs (L(k, j), j);
    //   backward kBNode: x(k) over U(k, r) from s0 + 1, rows pRows[first .. end); kBPair: x(k + 1) then x(k), U(k, r)
    //   from s0, U(k + 1, r) from s1, U(k, k + 1) at aux, rows P_{k+1}.
    // hasA bits: whether each output starts from a value of A (bit i for output i; the block's 4 outputs in the order
    // (k, k), (k, k + 1), (k + 1, k), (k + 1, k + 1)).
    struct PairSchedule {
        bool on = false;
        int nUnits = 0, nPaired = 0, nLevels = 0;
        std::vector<int32_t> taskA, taskB;  // factorisation and forward tasks, 4 ints each
        std::vector<int32_t> bTaskA, bTaskB;
        std::vector<int32_t> pairs;         // 2 per pair
        Schedule factor, backward, forward; // work: task indices (backward: into bTask*)
        std::vector<int32_t> unitOf, unitLevel, unitParent;  // node -> unit; per unit its level and parent unit (-1)
    };
    PairSchedule ps;

    // The top of the elimination tree (levels >= L0) held in shared memory by the one-system walks: the LU
    // values of its nodes (node k's [diag, U..., L...] from smemBase[k]) and then their right-hand-side values
    // (smem index yIdx[k]). Every pair of a top entry is internal (its node j is a top node: both operands in
    // shared memory, smem indices) or external (j below L0: global indices, applied in one parallel pass before
    // the top walk, as their operands are final by then). L0 is the lowest level whose top fits the budget;
    // built once per element size (FP64 / FP32).
    struct TopPart {
        int L0 = 0;                   // nLevels: no top part
        int nSlots = 0, nNodes = 0;   // smem LU values, then smem right-hand-side values
        std::vector<int32_t> smemBase, yIdx;   // per node (-1 below L0)
        std::vector<int32_t> slotGlobal;       // per smem LU value: its global LU slot
        std::vector<int32_t> slotDiagNode;     // per smem LU value: the node whose diagonal it is, else -1
        std::vector<int32_t> nodes;            // top nodes, smem right-hand-side order
        // all entries of the top nodes: the global entry, its smem index, internal and external pairs
        std::vector<int32_t> ent, entSm;
        std::vector<int32_t> intPtr, extPtr;   // [nEnt + 1]
        std::vector<int32_t> intPairs, extPairs;
        // load + external pass of the factorisation: all top entries (wide first); of the forward
        // substitution of a second right-hand side: the forward entries (wide first). Indices into ent.
        std::vector<int32_t> loadList, fwdLoadList;
        int loadWide = 0, fwdLoadWide = 0;
        // walks: per (level - L0) and phase, indices into ent, wide first; the forward entries per level;
        // the backward nodes per level (indices into nodes) with their U rows as smem right-hand-side indices
        std::vector<int32_t> fWalk, fWalkPtr, fWalkWide;   // ptr [2 * nTop + 1], wide [2 * nTop]
        std::vector<int32_t> vWalk, vWalkPtr, vWalkWide;   // ptr [nTop + 1]
        std::vector<int32_t> bWalk, bWalkPtr, bWalkWide;   // ptr [nTop + 1]
        std::vector<int32_t> bRowPtr, bRowSm;              // per top node (nodes order): smem indices of x(P_k)
        size_t bytes(size_t elem) const { return (size_t)(nSlots + nNodes) * elem; }
    };
    TopPart top[2];  // [0] FP64, [1] FP32
};

// The subtrees below a cut of the paired schedule's unit tree: every unit at level <= cut belongs to the subtree of
// its highest ancestor at level <= cut, and a subtree's tasks read only entries of its own units, so one CTA per
// (subtree, system group) can factor it alone, level by level with block barriers. Per subtree its stages (unit
// levels bottom-up, the two factorisation phases each, empty ones left out), each a range of factorisation work
// positions: stages of subtree t are subStage[t] .. subStage[t + 1] - 1, stage q holds work[stagePtr[q] ..
// stagePtr[q + 1]). Subtrees are ordered largest first (by task pairs).
struct SubtreeSchedule {
    int cut = -1;
    int nSub = 0;
    std::vector<int32_t> subStage, stagePtr, work;
    int64_t maxEntries = 0;     // LU entries of the largest subtree
    double pairShare = 0.0;     // share of the factorisation's pairs below the cut
};
SubtreeSchedule BuildSubtrees(const Symbolic& s, int cut);

// Build s.top[which] for values of `elem` bytes within `budget` bytes of shared memory.
void BuildTopPart(Symbolic& s, int which, size_t elem, size_t budget);

// Build the symbolic analysis; returns an empty string on success, else the reason.
std::string Analyze(const HostGrid& g, Symbolic& s, bool qlim = false);

// The static-pivot LU symbolic of s.m and the structurally symmetric pattern s.jRowPtr / s.jCol (diagonal present):
// minimum-degree order, LU pattern, levels, Crout entries and their index pairs, work schedules, top parts. mapA gets
// slotOf(k, l) (the LU slot of permuted cell (k, l), -1 outside the pattern) to record the caller's value maps, and
// marks the slots that receive a value of A (the rest are fill and start from zero).
std::string FactorSymbolic(Symbolic& s, const std::function<void(const std::function<int64_t(int, int)>&,
                                                                 std::vector<char>&)>& mapA);

// The symbolic analysis of a general square sparse matrix (CSR, n x n): the pattern of A + A^T with the diagonal,
// then FactorSymbolic. aSlot[q] is the LU slot of A's q-th stored entry (CSR order). Empty string on success.
std::string AnalyzeMatrix(int n, const int* rowPtr, const int* colIdx, Symbolic& s, std::vector<int>& aSlot);

// DC power-flow angles (degrees) of the grid with the branches `skip` out, referenced at bus `slack`, with the
// loads scaled by loadScale[i] (may be null); false unless the DC model is one island (gs_dc.cpp).
// For an element outage, `deadBus` is a removed bus (-1 none) and bus `specBus` (-1 none) loses specDpPu of generation.
bool DcAngles(const HostGrid& h, const Symbolic& s, const std::vector<int>& skip, int slack, const double* loadScale,
              std::vector<double>& thetaDeg, int deadBus = -1, int specBus = -1, double specDpPu = 0.0);

// Multi-branch outages (ContingencyAnalysis.ScreenOutageCore over several indices, :1087-1097). A set's outage id
// is nbr + its position in the table; one branch keeps its own index (the N-1 path). Per set: its branches (-1
// padded), the distinct Y cells they touch in ascending order (an INT_MAX sentinel after the last), and each cell's
// value summed without every branch of the set, in stamping order.
constexpr int kSetBranches = 16;  // a bus outage takes every branch at the bus
constexpr int kSetStride = 4 * kSetBranches + 1;
struct OutageSetTable {
    int n = 0;
    std::vector<int> br;      // [n * kSetBranches]
    std::vector<int> cell;    // [n * kSetStride]
    std::vector<double> red;  // [n * 2 * kSetStride] (G, B) per cell
};
// The per-system changes of an element outage (a generator or a bus, ScreenElementOutage,
// Analysis/ContingencyAnalysis.cs:1355-1437): up to two buses whose type changes (3 reference, 2 PV, 1 PQ, 0 removed)
// with the magnitude they hold or start from (NaN: as the grid), the bus that loses a unit with the lost output (pu)
// and the Q limits of its remaining units (MVAr).
struct ElemSys {
    int ovBus[2] = {-1, -1};
    int ovType[2] = {0, 0};
    double ovVm[2] = {NAN, NAN};
    int specBus = -1;
    double dp = 0.0, dq = 0.0, qmin = 0.0, qmax = 0.0;
};

// Append the set of in-service branches `b` (2..kSetBranches distinct indices); returns its position.
int AddOutageSet(const Symbolic& s, const std::vector<int>& b, OutageSetTable& t);

// Minimum-degree order of a structurally symmetric pattern (pivot step -> index).
std::vector<int> MinimumDegreeOrder(int n, const std::vector<int>& rowPtr, const std::vector<int>& col);

}  // namespace gs
