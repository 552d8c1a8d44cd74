// gs_kernels.cuh — device kernels of the gridsim_b200 batched Newton-Raphson engine (sm_100a).
//
// Layout: every per-system quantity is batch-interleaved, value[index * B + s], B a multiple of 32.
// A warp always works on 32 consecutive systems of one item (bus, LU entry, branch), so its loads and
// stores are single 128-byte (FP32) or 256-byte (FP64) transactions, and index data read by the warp is
// a broadcast. Systems are independent; no kernel synchronises across blocks.
#pragma once
#include <cstdint>

#include "gs_internal.h"

namespace gs {

// per-system flags
enum : int32_t {
    kFlagNonFinite = 1,       // the mismatch or the Jacobian held a NaN / Inf
    kFlagStepBad = 2,         // the step was not finite (NewtonShell.SolveStep refuses it)
    kFlagPivotPerturbed = 4,  // a static pivot fell below its floor and was perturbed
    kFlagJacBad = 8,          // the Jacobian held a NaN / Inf (the step is refused)
    kFlagPivoted = 16,        // solved with row partial pivoting (the re-solve of a collapsed static pivot)
    kFlagPivotFailed = 32,    // the partial-pivoting solve found the matrix singular (or out of capacity)
};

// Symbolic::TopPart on the device (one per element size).
struct DevTop {
    int L0, nSlots, nNodes, nEnt, loadWide, nLoad, fwdLoadWide, nFwdLoad;
    const int* slotGlobal;
    const int* slotDiagNode;
    const int* nodes;
    const int* smemBase;
    const int* ent;
    const int* entSm;
    const int* intPtr;
    const int* extPtr;
    const int2* intPairs;
    const int2* extPairs;
    const int* loadList;
    const int* fwdLoadList;
    const int* fWalk;
    const int* fWalkPtr;
    const int* fWalkWide;
    const int* vWalk;
    const int* vWalkPtr;
    const int* vWalkWide;
    const int* bWalk;
    const int* bWalkPtr;
    const int* bWalkWide;
    const int* bRowPtr;
    const int* bRowSm;
};

struct DevGrid {
    int n, m, nnzY, nbr;
    int64_t nnzLU;
    int nLevels;          // elimination-tree levels of the schedules
    int qlim;             // every bus has P and Q rows (identity rows where the bus is PV, reference or removed)
    int qlimOn;           // with qlim: PV buses switch to PQ at their Q limits (Q-limit enforcement)
    int qlimRevert;       // with qlimOn: a pinned bus may revert to PV in the pass that switches others
    int qlimMaxPasses;    // cap on switching passes
    double baseMva;
    const double* qminPu; // aggregate reactive limits per bus (pu)
    const double* qmaxPu;
    const double* qminMvar;
    const double* qmaxMvar;
    const int* yRowPtr;
    const int* yCol;
    const double* yG;
    const double* yB;
    const int* brCell;
    const double* brRed;
    const double* brStamp;
    const int* brF;
    const int* brT;
    const double* rateA;  // ratings / base (0 = unrated or not given)
    const double* rateB;
    const double* rateC;
    const uint8_t* brOn;
    int nSet;             // multi-branch outage sets of the current call (OutageSetTable; ids nbr .. nbr+nSet-1)
    const int* setBr;
    const int* setCell;
    const double* setRed;
    int nBnd;             // boundaries: members bndPtr[q] .. bndPtr[q+1]-1 (branch, direction), limit MW
    const int* bndPtr;
    const int* bndBranch;
    const int* bndDir;
    const double* bndLimit;
    const double* zip;    // [6 n] ZIP load coefficients per bus (Ap Bp Cp Aq Bq Cq), null: every load constant power
    const double* pgen;   // generation per bus (pu)
    const double* qgen;
    const double* pload;  // load per bus (pu)
    const double* qload;
    const double* vm0;
    const double* va0;
    const int* busType;   // effective type (1 PQ, 2 PV, 3 slack)
    const int* busP;
    const int* busQ;
    const int* ySlot;
    const int32_t* entSlot;
    const int32_t* entKind;
    const int32_t* entHasA;
    const int64_t* entPairPtr;
    const int2* pairs;
    const int32_t* diagEnt;
    const int* levelNodes;
    const int* levelNodePtr;
    const int32_t* entNode;
    // work schedules (see Symbolic::Schedule): factorisation, backward and forward substitution
    const int* fWork;
    const int* fItems;
    const int* fLevelPtr;
    const int* bWork;
    const int* bItems;
    const int* bLevelPtr;
    const int* vWork;
    const int* vItems;
    const int* vLevelPtr;
    const int* fWorkPtr;  // per level (and phase for the factorisation): work range
    const int* bWorkPtr;
    const int* vWorkPtr;
    const int4* fDesc;    // per schedule position: the work descriptor (see gs_engine.cu)
    const int4* bDesc;
    const int4* vDesc;
    const int* fMid;      // per level (phase): the mid-length short pieces after the wide ones
    const int* bMid;
    const int* vMid;
    const int* fWide;     // per level (phase): leading wide items
    const int* bWide;
    const int* vWide;
    const int64_t* luBase;
    const int* luCnt;
    const int* pRowPtr;
    const int* pRows;
    DevTop top[2];        // [0] FP64, [1] FP32
    // the paired schedule (Symbolic::PairSchedule): units of one node or a 2 x 2 pair; per schedule the task
    // descriptors A / B in schedule order, the items and the per-level (phase) item and work ranges
    int psLevels;         // 0: no paired schedule
    const int2* psPairs;
    const int4* pfA;
    const int4* pfB;
    const int* pfItems;
    const int* pfLevelPtr;
    const int* pfWorkPtr;
    const int* pfWide;
    const int* pfMid;
    const int4* pbA;
    const int4* pbB;
    const int* pbItems;
    const int* pbLevelPtr;
    const int* pbWorkPtr;
    const int* pbWide;
    const int* pbMid;
    const int4* pvA;
    const int4* pvB;
    const int* pvItems;
    const int* pvLevelPtr;
    const int* pvWorkPtr;
    const int* pvWide;
    const int* pvMid;
};

struct DevBatch {
    int B;                  // interleave stride (multiple of 32)
    int count;              // live systems
    int nLevels;            // elimination-tree levels of the grid
    double* vm;             // [n][B]
    double* va;             // [n][B]
    void* lu;               // [nnzLU][B] of the LU type (diagonal slots keep A(k, k))
    void* piv;              // [m][B] pivots U(k, k)
    void* y;                // [m][B] right-hand side / step
    void* z;                // [m][B] correction (mixed precision), or null
    double* rhs64;          // [m][B] FP64 mismatch (mixed precision), or null
    int* refine;            // [B] refine this step (mixed precision), or null
    unsigned long long* maxMis;  // [B] bit pattern of a non-negative double
    unsigned long long* maxDx;
    double* startMis;       // [B] mismatch at the start of the current Newton run
    double* beforeLast;     // [B] mismatch the last step was taken from (the DC retry's stall test)
    double* finalMis;       // [B]
    int* status;            // [B]
    int* iters;             // [B] steps taken
    int* convIters;         // [B] steps taken when the tolerance was first met
    int* active;            // [B]
    int* flags;             // [B]
    const int* outage;      // [B] branch index or -1
    const double* loadScale;  // [n][B] or null
    int* activeCount;       // [2]: systems still stepping, of which refine their step (mixed precision)
    int* activeList;        // [B] systems still stepping (filled for the few-systems path)
    // Q-limit enforcement (grids with qlim), else null
    int* effType;           // [n][B] the bus's type now (2 PV, 1 switched to PQ), for buses that start PV
    double* qspecSys;       // [n][B] Q specification of a switched bus (pu)
    int* pinned;            // [n][B] 0 none, 1 at Qmax, -1 at Qmin, 2 fixed (Qmin == Qmax)
    int* reverted;          // [n][B] reverts to PV so far
    double* qinj;           // [n][B] Q injection at the last mismatch (pu)
    int* passIter;          // [B] steps of the current Q-limit pass
    int* qPass;             // [B] passes completed
    int* qState;            // [B] kQ* bits
    // element outages (grids with qlim: every bus has P and Q rows), else null: per system up to two buses whose
    // type changes (3 reference, 2 PV, 1 PQ, 0 removed) with the magnitude they start from or hold (NaN: as the
    // grid), and the bus that loses units with the generation it loses (pu) and its remaining Q limits (MVAr)
    const int* ovBus;       // [2B] bus or -1
    const int* ovType;      // [2B]
    const double* ovVm;     // [2B]
    const int* specBus;     // [B] bus or -1
    const double* specDp;   // [B]
    const double* specDq;   // [B]
    const double* specQmin; // [B]
    const double* specQmax; // [B]
};

// qState bits
enum : int32_t { kQPending = 1, kQChanged = 2, kQSkipStep = 4, kQFinalPass = 8, kQFinalConverged = 32 };

// The Y cells a system's outage changes, walked in step with a row's cells: one branch (its four cells and their
// values without it, brCell / brRed) or an outage set (its distinct cells in ascending order and their values without
// every branch of the set). Construct with the row's first cell; call at() for each cell of the row in order.
struct CellOverride {
    int o, c0, c1, c2, c3, ov;
    const int* sc;
    const double* sr;
    __device__ __forceinline__ CellOverride(const DevGrid& g, int outage, int p0)
        : o(outage), c0(-1), c1(-1), c2(-1), c3(-1), ov(0), sc(nullptr), sr(nullptr) {
        if (o >= g.nbr) {
            const int q = o - g.nbr;
            sc = g.setCell + (size_t)kSetStride * q;
            sr = g.setRed + (size_t)2 * kSetStride * q;
            while (sc[ov] < p0) ov++;  // stops at the sentinel
        } else if (o >= 0) {
            c0 = g.brCell[4 * o]; c1 = g.brCell[4 * o + 1]; c2 = g.brCell[4 * o + 2]; c3 = g.brCell[4 * o + 3];
        }
    }
    __device__ __forceinline__ void at(const DevGrid& g, int p, double& G, double& Bv) {
        if (p == c0) { G = g.brRed[8 * o + 0]; Bv = g.brRed[8 * o + 1]; }
        else if (p == c1) { G = g.brRed[8 * o + 2]; Bv = g.brRed[8 * o + 3]; }
        else if (p == c2) { G = g.brRed[8 * o + 4]; Bv = g.brRed[8 * o + 5]; }
        else if (p == c3) { G = g.brRed[8 * o + 6]; Bv = g.brRed[8 * o + 7]; }
        else if (sc && p == sc[ov]) { G = sr[2 * ov]; Bv = sr[2 * ov + 1]; ov++; }
    }
};

// True when branch k is out in a system whose outage id is o.
__device__ __forceinline__ bool branchOut(const DevGrid& g, int o, int k) {
    if (o < g.nbr) return o == k;
    const int* br = g.setBr + (size_t)kSetBranches * (o - g.nbr);
    for (int j = 0; j < kSetBranches && br[j] >= 0; j++)  // -1 after the last
        if (br[j] == k) return true;
    return false;
}

}  // namespace gs
